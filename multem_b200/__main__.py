"""Run a MULTEM simulation stored in a MAT-file: python -m multem_b200 IN.mat OUT.mat [--var NAME] [--compress]

IN.mat holds the struct of multem_input.parameters.toStruct (saved from MATLAB with `save`, -v6 or
-v7); OUT.mat receives `output_multislice` as ilc_multem returns it."""
import argparse

from . import api


def main():
    ap = argparse.ArgumentParser(prog="python -m multem_b200", description=__doc__.splitlines()[0])
    ap.add_argument("input")
    ap.add_argument("output")
    ap.add_argument("--var", default=None, help="input variable (default: the first struct in the file)")
    ap.add_argument("--compress", action="store_true", help="write -v7 (zlib) elements")
    a = ap.parse_args()
    api.ilc_multem_mat(a.input, a.output, a.var, a.compress)


if __name__ == "__main__":
    main()
