"""Close-packed lattice of the reference's cases (src/cases/lattice.py:4-34).

Layers stacked in z with period three, rows in y alternating by half a
spacing in x, the reference's counts (rounded down to even rows and
multiples of three layers) and offsets: the same points the reference's case
generators start from (checked against fixtures from the reference's own
function in tests/test_cases_cpu.py).
"""

import numpy as np


def _count(extent, pitch):
    return int(np.ceil(np.nextafter(extent / pitch, -np.inf)))


def close_packed_lattice(bounds, spacing):
    xmin, xmax, ymin, ymax, zmin, zmax = bounds
    row_pitch = spacing * np.sqrt(3.0 / 4.0)
    layer_pitch = spacing * np.sqrt(6.0) / 3.0
    nx = _count(xmax - xmin, spacing)
    ny = 2 * (_count(ymax - ymin, row_pitch) // 2)
    nz = 3 * (_count(zmax - zmin, layer_pitch) // 3)
    dx, dy, dz = (xmax - xmin) / nx, (ymax - ymin) / ny, (zmax - zmin) / nz
    col, row, layer = np.meshgrid(np.arange(nx), np.arange(1, ny + 1), np.arange(1, nz + 1), indexing="ij")
    odd_row = row % 2 == 1
    phase = layer % 3
    # half-spacing shift in x: layers 0 and 1 on even rows, layer 2 on odd rows
    shift_x = np.where(((phase == 0) | (phase == 1)) & ~odd_row, 0.5, 0.0)
    shift_x = np.where((phase == 2) & odd_row, 0.5, shift_x)
    shift_y = np.select([phase == 0, phase == 2], [2.0 / 3.0, 1.0 / 3.0], 0.0)
    x = xmin + 0.25 * spacing + (col + shift_x) * dx
    y = ymin + (row - 1.0 + 1.0 / 6.0 + shift_y) * dy
    z = zmin + (layer - 0.5) * dz
    return x.ravel(), y.ravel(), z.ravel()
