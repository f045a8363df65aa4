"""Stage the reference's published large instances for the GPU tests.

The reference ships the instances its reports were measured on
(examples/vsli/*.tsp, examples/art/*.tsp).  The GPU tests that check the CUDA
path against those published values (tests/test_published_scale.py) read
gzip copies of them from tests/golden/_instances/, a folder that is not
committed (the instances are the reference's data) but travels with the
working tree.  This script fills it from a local reference checkout
(argument 1; default $F2M_REFERENCE, else a sibling checkout named
"reference" next to this repository); __graft_entry__.build() runs it.

  python tests/golden/stage_instances.py [reference_dir]
"""
import gzip
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_instances")
FILES = ["examples/vsli/ara238025.tsp", "examples/vsli/sra104815.tsp",
         "examples/art/mona-lisa100K.tsp", "examples/art/vangogh120K.tsp",
         "examples/art/venus140K.tsp", "examples/art/pareja160K.tsp",
         "examples/art/courbet180K.tsp"]


def reference_dir():
    root = os.path.dirname(os.path.dirname(HERE))
    return os.environ.get("F2M_REFERENCE") or os.path.join(os.path.dirname(root), "reference")


def stage(ref=None):
    ref = ref or reference_dir()
    if not os.path.isdir(ref):
        return 0
    os.makedirs(OUT, exist_ok=True)
    n = 0
    for rel in FILES:
        src = os.path.join(ref, rel)
        dst = os.path.join(OUT, os.path.basename(rel) + ".gz")
        if not os.path.exists(src):
            continue
        if os.path.exists(dst) and os.path.getmtime(dst) >= os.path.getmtime(src):
            n += 1
            continue
        with open(src, "rb") as f, gzip.open(dst + ".part", "wb", compresslevel=6) as g:
            shutil.copyfileobj(f, g)
        os.replace(dst + ".part", dst)
        n += 1
    return n


if __name__ == "__main__":
    print(f"staged {stage(sys.argv[1] if len(sys.argv) > 1 else None)} instances in {OUT}")
