"""Generates the golden fixtures in tests/golden/ from the reference's OWN code.

Run where the reference tree is available, after `make -C oracle REF=<tree>`:

    python tests/golden/make_golden.py --ref <root of the reference tree>

* ref_sbr.npz -- for every small case below: the field per (angle, frequency)
  and the per-ray hit records (hitCount, hitDist) of the reference's per-ray
  routine src/cuda/rtKernels.cu and BVH builder src/scene/bvhBuilder.cpp,
  compiled for the host in FP64 (-DUSE_DOUBLE) into oracle/_ref by oracle/Makefile,
  with the PO term restated from src/cuda/poKernels.cu:81-109.
* mie_ref.json -- sigma/(pi r^2) from the reference's normalized_rcs
  (util/monostatic_PEC_sphere.py:8-58), executed from its source with only that
  function compiled (the script's module-level plotting code is skipped).

The meshes are the seeded synthetic generators of sagittasbr_b200.meshes, so the
fixture inputs are reproducible without the reference.
"""
from __future__ import annotations

import argparse
import ast
import json
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from sagittasbr_b200 import meshes as M  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def cases():
    """name -> (verts, tris, theta, phi, freqs, nx, ny, G, max_bounces, R)."""
    out = {}
    v, t = M.box(1.0)
    out["box"] = (v, t, [90.0, 45.0, 30.0, 0.0, 120.0], [0.0, 45.0, 10.0, 0.0, 200.0], [1e9, 3e9], 24, 24,
                  2.0 * M.bounding_radius(v), 5, 1.0)
    v, t = M.icosphere(2, 1.0)
    out["ico2"] = (v, t, [90.0, 90.0, 60.0, 10.0], [0.0, 33.0, 71.0, 5.0], [1e9, 2.5e9], 24, 24, 2.0, 3, 1.0)
    v, t = M.trihedral(1.0, 4)
    out["trihedral4"] = (v, t, [54.7356103172, 30.0, 80.0, 45.0, 0.0], [45.0, 20.0, 70.0, 0.0, 0.0], [1e10],
                         32, 32, 2.0 * M.bounding_radius(v), 3, 1.0)
    v, t = M.dihedral(1.0, 3)
    out["dihedral3"] = (v, t, [90.0, 90.0, 60.0], [45.0, 10.0, 45.0], [3e9, 1e10], 20, 20,
                        2.0 * M.bounding_radius(v), 4, 0.9)
    v, t = M.plate(1.0, 2)
    out["plate"] = (v, t, [0.0, 10.0, 30.0], [0.0, 0.0, 45.0], [5e9], 32, 32, 1.5, 2, 1.0)
    return out


def reference_mie(ref_root: str):
    src = open(os.path.join(ref_root, "util", "monostatic_PEC_sphere.py")).read()
    tree = ast.parse(src)
    fn = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "normalized_rcs"][0]
    mod = ast.Module(body=[fn], type_ignores=[])
    from scipy.special import spherical_jn, spherical_yn
    ns = {"np": np, "spherical_jn": spherical_jn, "spherical_yn": spherical_yn}
    exec(compile(mod, "monostatic_PEC_sphere.normalized_rcs", "exec"), ns)
    return ns["normalized_rcs"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference tree")
    a = ap.parse_args()
    O.build()
    if not O.ref_available(64):
        raise SystemExit("oracle/_ref not built: run make -C oracle with the reference present")
    blob = {}
    for name, (v, t, th, ph, fr, nx, ny, G, mb, R) in cases().items():
        out = O.ref_sweep(v, t, th, ph, fr, nx, ny, G, mb, R, kind=64, records=True, threads=4)
        blob[f"{name}/field"] = out.field
        blob[f"{name}/count"] = out.rays["count"].astype(np.int8)
        blob[f"{name}/dist"] = out.rays["dist"]
        print(name, "sigma", out.sigma.ravel()[:4], "hit frac", float((out.rays["count"] > 0).mean()))
    np.savez_compressed(os.path.join(HERE, "ref_sbr.npz"), **blob)

    f = reference_mie(a.ref)
    xs = [0.5, 1.0, 2.0, 5.0, 10.0, 20.9584502, 30.0, 100.0, 104.79, 209.58, 500.0, 999.0, 1000.0, 2000.0]
    json.dump({"x": xs, "normalized_rcs": [float(f(x)) for x in xs],
               "source": "util/monostatic_PEC_sphere.py:8-58 (normalized_rcs)"},
              open(os.path.join(HERE, "mie_ref.json"), "w"), indent=1)
    print("wrote", os.path.join(HERE, "ref_sbr.npz"), os.path.join(HERE, "mie_ref.json"))


if __name__ == "__main__":
    main()
