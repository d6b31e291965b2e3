"""``python -m tenes_b200 input.toml``: the ``tenes`` command (src/main.cpp:28-105)
for simple-update ground-state and time-evolution runs on the GPU path."""

import argparse
import sys

from .input import InputError
from .saveload import LoadError


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="tenes_b200", description="iTPS simple update + CTMRG on a B200")
    ap.add_argument("input", help="expert-format input.toml (as for tenes)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--mixed", action="store_true",
                    help="tensor-core mixed precision for the environment contractions")
    ap.add_argument("--outdir", default=None, help="override parameter.general.output")
    ap.add_argument("--quiet", action="store_true")
    a = ap.parse_args(argv)
    from .itps import run
    try:
        run(a.input, device=a.device, mixed=a.mixed, print_level=0 if a.quiet else 1, outdir=a.outdir)
    except (InputError, LoadError) as e:
        print(f"ERROR: {e}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
