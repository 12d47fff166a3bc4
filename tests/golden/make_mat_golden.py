"""Copies the reference's two ANTs-written 0GenericAffine-style .mat files into tests/golden/.

crates/fastwarp-reg/tests/data/ms0.mat and ms20.mat are MATLAB v4 files of 193 bytes that ANTs
wrote during the reference's development (an AffineTransform_double_3_3 with its fixed centre);
the reference's tests decode them independently and require its writer to reproduce them byte
for byte (crates/fastwarp-reg/tests/samples.rs:34-67). They hold transform parameters only. This
script copies the bytes unchanged; run it where the reference checkout is available:

    python tests/golden/make_mat_golden.py /path/to/fastwarp
"""
import os
import shutil
import sys

NAMES = ["ms0.mat", "ms20.mat"]


def main(ref_root):
    src = os.path.join(ref_root, "crates", "fastwarp-reg", "tests", "data")
    here = os.path.dirname(os.path.abspath(__file__))
    for name in NAMES:
        out = os.path.join(here, "ants_" + name)
        shutil.copyfile(os.path.join(src, name), out)
        print(f"wrote {out}: {os.path.getsize(out)} bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the fastwarp checkout>")
    main(sys.argv[1])
