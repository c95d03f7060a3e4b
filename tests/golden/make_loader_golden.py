"""Generates tests/golden/loader_ref.json from the reference's OWN model loader.

Run where the reference tree is available, after `make -C oracle REF=<tree>`:

    python tests/golden/make_loader_golden.py --ref <root of the reference tree>

For every model the reference ships in assets/test_models: the triangle count and
the SHA-256 of the de-indexed FP32 triangles (9 floats per triangle, little endian)
that src/modelLoader.cpp + runRcsApp's de-indexing (src/app/rtRcsEntry.cu:108-145)
produce at model scale 1 and 0.37.
"""
import argparse
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from oracle import oracle as O  # noqa: E402

SCALES = (1.0, 0.37)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference tree")
    a = ap.parse_args()
    models = os.path.join(a.ref, "assets", "test_models")
    out = {}
    for name in sorted(os.listdir(models)):
        if not name.endswith(".obj"):
            continue
        entry = {}
        for s in SCALES:
            tri = O.ref_load_triangles(os.path.join(models, name), s)
            entry[f"{s:g}"] = {"triangles": int(tri.shape[0]),
                               "sha256": hashlib.sha256(tri.astype("<f4").tobytes()).hexdigest()}
        out[name] = entry
    with open(os.path.join(HERE, "loader_ref.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"wrote {len(out)} models")


if __name__ == "__main__":
    main()
