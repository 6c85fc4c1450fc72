"""The C-ABI library loads and exports every symbol ``include/*.h`` declares.

Runs without a GPU: only symbol lookup and the pure-host entry points
(version, field-name tables) are called.
"""

import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))


def _declared():
    names = []
    for h in HEADERS:
        text = open(h).read()
        names += re.findall(r"^\s*(?:int|int32_t|int64_t|const char\*|void)\s+\**(mhd_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def _xmacro_fields():
    text = open(os.path.join(ROOT, "include", "mhd_b200.h")).read()
    out = []
    for macro in ("MHD_STATE_REQUIRED", "MHD_STATE_OPTIONAL"):
        body = re.search(r"#define " + macro + r"\(X\)((?:.*\\\n)*.*)", text).group(1)
        out += re.findall(r"X\((\w+)\)", body)
    return out + ["itype"]


@pytest.fixture(scope="module")
def lib():
    from src import _abi

    import build as pkg_build

    pkg_build.build()
    return _abi.load()


def test_every_declared_symbol_is_exported(lib):
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"symbols declared but not exported: {missing}"


def test_binding_covers_the_header(lib):
    from src import _abi

    assert sorted(_abi.EXPORTS) == _declared()


def test_state_layout_matches_header(lib):
    from src import _abi

    assert lib.mhd_abi_version() == 1
    assert _abi.STATE_FIELDS == _xmacro_fields()
    assert set(_abi.SORTED_FIELDS) <= set(_abi.STATE_FIELDS)
    assert _abi.SORTED_FIELDS[-1] == "itype"


def test_state_names_are_reference_property_names(lib):
    from src import _abi
    from src.particles import property_names

    assert set(_abi.STATE_FIELDS) <= set(property_names())


def test_context_creation_without_gpu_fails_loudly(lib):
    import torch

    from src import _abi

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = _abi.make_params(3, "cubic", 1.2, 5 / 3, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, [0, 0, 0], [1, 1, 1],
                         [True] * 3)
    ctx = ctypes.c_void_p()
    rc = lib.mhd_ctx_create(ctypes.byref(p), 16, ctypes.byref(ctx))
    assert rc == -6  # MHD_ERR_NO_DEVICE
