"""Command line: ``python -m src.run <config.toml>`` (src/run.py:32-39)."""

import argparse
from pathlib import Path

from .cases.alfven import AlfvenWave, AlfvenWave2D
from .cases.jadvect import CurrentLoopAdvection
from .cases.jet import JMXJets
from .cases.mhdblast import MHDBlast, MHDBlast3D
from .cases.mhdrotor import MHDRotor
from .cases.mhdshock import MHDShock, MHDShock2D
from .cases.mhdsine import MHDSine
from .cases.mhdvortex import MHDVortex
from .cases.mhdwave import MHDWave
from .cases.orstang import OrszagTang, OrszagTang2D
from .config import load_config

# the reference's case names (src/run.py:16-29) and the benchmark's forms
CASES = {
    "1jet": JMXJets,
    "3jet": JMXJets,
    "12jet": JMXJets,
    "alfven": AlfvenWave,
    "alfven2d": AlfvenWave2D,
    "jadvect": CurrentLoopAdvection,
    "mhdblast": MHDBlast,
    "mhdblast3d": MHDBlast3D,
    "mhdrotor": MHDRotor,
    "mhdshock": MHDShock,
    "mhdshock2d": MHDShock2D,
    "mhdsine": MHDSine,
    "mhdvortex": MHDVortex,
    "mhdwave": MHDWave,
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
