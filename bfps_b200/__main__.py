"""Command line: `python -m bfps_b200 DNS NSVEparticles -n 32 ...`, the
counterpart of `bfps DNS NSVEparticles ...` (bfps/__main__.py:18-110) for
the NSVE / NSVEparticles path; the reference's other base classes (PP,
TEST, NavierStokes, FluidResize, ...) are not part of this package."""
import argparse
import sys

from .dns import DNS, VERSION


def main(argv=None):
    argv = sys.argv[1:] if argv is None else list(argv)
    parser = argparse.ArgumentParser(prog="bfps_b200")
    parser.add_argument("-v", "--version", action="version", version="%(prog)s " + VERSION)
    parser.add_argument("base_class", choices=["DNS"], type=str)
    opt = parser.parse_args(argv[:1])
    if opt.base_class == "DNS":
        DNS().launch(argv[1:])


if __name__ == "__main__":
    main()
