"""Copies FlowLB's example inputs and their mesh.vti files into
tests/golden/setup/<case>/ as the fixtures of the file-based set-up tests.

Source: the reference tree's test/ejemplos/<case>/{Geometry.txt,
OptionsCalc.txt, mesh.vti}.  mesh.vti is what FlowLB's App::createDomain
wrote for that case (geometry flags after the free-surface sweep); it is
stored gzip-compressed (mtime 0) and compared byte for byte.

Four of the committed mesh.vti files were written from earlier versions of
their input files.  The values below restore those versions; each one is read
off the mesh.vti itself (its WholeExtent, Spacing and boundary flags):

* damBreak: the fluid column spans rows 10..60 of 101 (y 0.10..0.60 m at
  0.01 m), i.e. INITIAL_CONDITION_FLAG(1).height 0.5 about its centre 0.35.
* cavity: Spacing 0.001 (SIZE), the INLET row is the top one and the left
  column is WALL (LEFT_BOUNDARY WALL, UP_BOUNDARY INPUT).
* Poiseuille_plano: WholeExtent 0..4000 at Spacing 0.005 (x length 20 m,
  SIZE 0.005); INLET and OUTLET columns (LEFT INPUT, RIGHT OUTPUT).
* modulos: WholeExtent 0..2000 x 0..600 at 0.01 (x length 20 m, domain
  height 6 m from a CDW radius of 3).

The remaining examples (coche, pantalon, plenum) hold flags in an older
encoding (values 0, 6 and 9) and options the current reader rejects; they are
not used.

Usage: python tests/golden/make_setup_fixtures.py --ref /path/to/FlowLB   (or FLOWLB_REF=/path/to/FlowLB)
"""
from __future__ import annotations

import argparse
import gzip
import os

HERE = os.path.dirname(os.path.abspath(__file__))

OVERRIDES = {
    "damBreak": {
        "OptionsCalc.txt": [("INITIAL_CONDITION_FLAG(1).height = 0.8", "INITIAL_CONDITION_FLAG(1).height = 0.5")],
    },
    "cavity": {
        "Geometry.txt": [("SIZE = 0.01", "SIZE = 0.001")],
        "OptionsCalc.txt": [("LEFT_BOUNDARY = INPUT", "LEFT_BOUNDARY = WALL"),
                            ("UP_BOUNDARY = WALL", "UP_BOUNDARY = INPUT")],
    },
    "Poiseuille_plano": {
        "Geometry.txt": [("POINT(2) = (10, 0, 0)", "POINT(2) = (20, 0, 0)"), ("SIZE = 0.0005", "SIZE = 0.005")],
        "OptionsCalc.txt": [("LEFT_BOUNDARY = PERIODIC", "LEFT_BOUNDARY = INPUT"),
                            ("RIGHT_BOUNDARY = PERIODIC", "RIGHT_BOUNDARY = OUTPUT")],
    },
    "modulos": {
        "Geometry.txt": [("POINT(2) = (15, 0, 0)", "POINT(2) = (20, 0, 0)"),
                         ("CDW(1).radius = 2.5", "CDW(1).radius = 3")],
    },
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("FLOWLB_REF"),
                    help="FlowLB source tree (default: $FLOWLB_REF)")
    a = ap.parse_args()
    if not a.ref:
        ap.error("give the FlowLB source tree with --ref or FLOWLB_REF")
    for case, subs in OVERRIDES.items():
        src = os.path.join(a.ref, "test", "ejemplos", case)
        dst = os.path.join(HERE, "setup", case)
        os.makedirs(dst, exist_ok=True)
        for fn in ("Geometry.txt", "OptionsCalc.txt"):
            text = open(os.path.join(src, fn), encoding="utf-8").read()
            for old, new in subs.get(fn, []):
                if old not in text:
                    raise SystemExit(f"{case}/{fn}: '{old}' not found")
                text = text.replace(old, new)
            with open(os.path.join(dst, fn), "w", encoding="utf-8") as f:
                f.write(text)
        raw = open(os.path.join(src, "mesh.vti"), "rb").read()
        with open(os.path.join(dst, "mesh.vti.gz"), "wb") as f:
            f.write(gzip.compress(raw, compresslevel=9, mtime=0))
        print(case, len(raw), "bytes of mesh.vti")


if __name__ == "__main__":
    main()
