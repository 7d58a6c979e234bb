"""Regenerates the golden fixtures in this folder from the reference tree.

dm2000.list is the reference's only shipped golden vector (Share/dm2000.list):
the DM trials of its dedisp generator for the default search setup.  It is
copied verbatim; nothing else is derived here.  Run from the repository root
with the reference tree's location as the argument (or in HEIMDALL_REFERENCE):

    python tests/golden/make_golden.py <path to the reference tree>
"""
import os
import shutil
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HEIMDALL_REFERENCE")
if not ref:
    sys.exit("usage: make_golden.py <path to the reference tree>")
here = os.path.dirname(os.path.abspath(__file__))
shutil.copyfile(os.path.join(ref, "Share", "dm2000.list"), os.path.join(here, "dm2000.list"))
print("wrote", os.path.join(here, "dm2000.list"))
