"""Command line of the reference's main.py (nh-flood-2d main.py:1-21):

    python -m nhflood --domain domain.json --force force.json

runs ``run_simulation`` on the two configs. ``--pipe`` is accepted for the
same command line, but SWMM pipe coupling is not part of this engine, so a
pipe config is refused before any work starts.
"""
from __future__ import annotations

import argparse

from .input import load_domain_config, load_force_config
from .solver_compact import run_simulation


def main(argv=None) -> None:
    parser = argparse.ArgumentParser(prog='python -m nhflood', description='Run the configured two-dimensional model.')
    parser.add_argument('--domain', required=True, help='Domain JSON configuration')
    parser.add_argument('--force', required=True, help='Boundary/rainfall JSON configuration')
    parser.add_argument('--pipe', help='Optional SWMM pipe configuration (not supported by this engine)')
    args = parser.parse_args(argv)
    if args.pipe:
        parser.error('SWMM pipe coupling is not part of this engine')
    run_simulation(load_domain_config(args.domain), load_force_config(args.force))


if __name__ == '__main__':
    main()
