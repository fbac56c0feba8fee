"""The reference's own dumps of an assembled system (UMFPackMatrix::dump /
UMFPackVector::dump, src/linsolver/umfpack.cc:95-127, 194-220) in its binary
(H2DX / H2DR) and MATLAB formats, written by the reference (oracle/_ref,
driver option --dump) for the c1_small fixture's problem:

    make -C oracle && python tests/golden/make_dump_golden.py

Writes tests/golden/dump/c1_small.{h2dx,h2dr,m}.
"""
from __future__ import annotations

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from hermes3d_b200.mesh import unit_cube  # noqa: E402
from oracle import ref_driver  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dump")


def main():
    if not ref_driver.available():
        ref_driver.build()
    os.makedirs(OUT, exist_ok=True)
    # the c1_small case of make_golden.py
    r = ref_driver.run(unit_cube(2), p=3, qmode="fixed:5", source="one", bc="dirichlet0",
                       dump=os.path.join(OUT, "c1_small"))
    print("c1_small ndof", r["ndof"], "nnz", r["nnz"])


if __name__ == "__main__":
    main()
