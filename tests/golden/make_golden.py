"""Copies the reference's shipped golden outputs and sample inputs into this
directory as test fixtures (run once, with the path of a checkout of the
reference as the only argument; the fixtures are committed, so tests never
read the reference).

Usage: python tests/golden/make_golden.py <reference project root>

Sources, relative to the reference project root:
  input/imag3d-input, input/real3d-input            parameter files
  output/imag3d-mpicuda/imag3d-{out,rms}.txt         printed rows (16 ranks)
  output/imag3d-mpicuda/imag3d-den1d_{x,y,z}.bin     full-precision profiles
  output/real3d-mpicuda/real3d-{out,rms,dyna}.txt
  output/real3d-mpicuda/real3d-den1d_{x,y,z}.bin
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

FILES = [
    ("input/imag3d-input", "imag3d-input"),
    ("input/real3d-input", "real3d-input"),
    ("output/imag3d-mpicuda/imag3d-out.txt", "imag3d-out.txt"),
    ("output/imag3d-mpicuda/imag3d-rms.txt", "imag3d-rms.txt"),
    ("output/real3d-mpicuda/real3d-out.txt", "real3d-out.txt"),
    ("output/real3d-mpicuda/real3d-rms.txt", "real3d-rms.txt"),
    ("output/real3d-mpicuda/real3d-dyna.txt", "real3d-dyna.txt"),
] + [("output/imag3d-mpicuda/imag3d-den1d_%s.bin" % a, "imag3d-den1d_%s.bin" % a) for a in "xyz"] \
  + [("output/real3d-mpicuda/real3d-den1d_%s.bin" % a, "real3d-den1d_%s.bin" % a) for a in "xyz"]

if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <reference project root>")
    REF = sys.argv[1]
    for src, dst in FILES:
        shutil.copyfile(os.path.join(REF, src), os.path.join(HERE, dst))
        print(dst)
