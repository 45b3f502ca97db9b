"""``lbm`` command: run a YAML case (the reference's ``lbm`` entry point, src/LBM/cli.py:9-40).

    python -m lbm_porouschem_b200 -c config.yaml [-v 0|1|2] [--max-steps N]
"""
from __future__ import annotations

import argparse
import logging
import os
import sys


def run(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="lbm", description="run a lattice-Boltzmann case from a YAML file")
    ap.add_argument("--config", "-c", default="config.yaml", help="the configuration of the simulation case")
    ap.add_argument("--verbose", "-v", type=int, default=1, help="log level 0:warning 1:info 2:debug")
    ap.add_argument("--max-steps", type=int, default=None, help="stop after this many lattice steps")
    args = ap.parse_args(argv)
    logger = logging.getLogger("LBM 2D logger")
    if not logger.handlers:
        logger.addHandler(logging.StreamHandler(sys.stdout))
    logger.setLevel({0: logging.WARNING, 1: logging.INFO, 2: logging.DEBUG}[args.verbose])
    path = args.config
    if not os.path.exists(path):
        found = [p for p in sorted(os.listdir(os.curdir)) if p.endswith(".yaml")]
        if not found:
            raise ValueError("The configuration file does not exist. Pass it with -c or create config.yaml.")
        logger.info(f"{path} not found. Found {found[0]} yaml file instead.")
        path = found[0]
    import yaml
    with open(path, "r", encoding="utf8") as f:
        logger.info(f"Loading {path} file")
        config = yaml.safe_load(f)
    from .app import application
    lb = application(config, logger, max_steps=args.max_steps)
    lb.close()
    return 0


if __name__ == "__main__":
    sys.exit(run())
