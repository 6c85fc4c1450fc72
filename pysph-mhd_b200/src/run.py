"""Command line: ``python -m src.run <config.toml>`` (src/run.py:32-39)."""

import argparse
from pathlib import Path

from .cases.alfven import AlfvenWave, AlfvenWave2D
from .cases.mhdblast import MHDBlast, MHDBlast3D
from .cases.mhdshock import MHDShock, MHDShock2D
from .cases.orstang import OrszagTang, OrszagTang2D
from .config import load_config

CASES = {
    "alfven": AlfvenWave,
    "alfven2d": AlfvenWave2D,
    "mhdblast": MHDBlast,
    "mhdblast3d": MHDBlast3D,
    "mhdshock": MHDShock,
    "mhdshock2d": MHDShock2D,
    "orstang": OrszagTang,
    "orstang2d": OrszagTang2D,
}


def main(argv=None):
    parser = argparse.ArgumentParser()
    parser.add_argument("config", type=Path)
    args = parser.parse_args(argv)
    config_types = {name: app.config_type for name, app in CASES.items()}
    config = load_config(args.config, config_types)
    application = CASES[config.case.name](config)
    pa = application.run()
    return application, pa


if __name__ == "__main__":
    main()
