"""Converts the reference's ITK 5.4.5 dense Mattes MI fixtures into tests/golden/mattes_itk.npz.

The fixtures (WyssCenter/fastwarp, crates/fastwarp-reg/tests/data/mattes/*.txt, written there by
scripts/itk_fixtures/mattes_fixtures.py with ITK's MattesMutualInformationImageToImageMetricv4 and
a DisplacementFieldTransform) hold `key: values` lines: grids, images, masks, the field, and
ITK's value, valid-point count and per-voxel derivative. This script only re-packs the numbers;
run it where the reference checkout is available:

    python tests/golden/make_golden.py /path/to/fastwarp
"""
import os
import sys

import numpy as np

NAMES = ["oblique_b12", "oblique_b32", "oblique_b32_masked", "virtual_b32",
         "virtual_b32_masked", "virtual_b32_masked_swapped"]


def load(path):
    out = {}
    with open(path) as fh:
        for line in fh:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            key, values = line.split(":", 1)
            out[key] = np.array([float(v) for v in values.split()], dtype=np.float64)
    return out


def main(ref_root):
    data_dir = os.path.join(ref_root, "crates", "fastwarp-reg", "tests", "data", "mattes")
    arrays = {}
    for name in NAMES:
        for key, v in load(os.path.join(data_dir, name + ".txt")).items():
            arrays[f"{name}/{key}"] = v
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mattes_itk.npz")
    np.savez_compressed(out, **arrays)
    print(f"wrote {out}: {len(arrays)} arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the fastwarp checkout>")
    main(sys.argv[1])
