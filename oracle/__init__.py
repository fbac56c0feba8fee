"""Test infrastructure: the C restatement (port) and the reference build
(ref_driver).  Only tests/, __graft_entry__ and bench.py's CPU-baseline and
reference legs use it; the product package never does."""
import os as _os

# Location of the reference sources (read only by the recipes that build the
# oracle and generate fixtures); HERMES3D_REF overrides the default.
REFERENCE_DIR = _os.environ.get("HERMES3D_REF", "/root/reference")
