"""Exact ties on the GPU: a mesh that holds triangles twice with opposite windings.

Where two coincident faces are hit at exactly the same distance, the reference keeps
the one its walk tests last (src/cuda/rtKernels.cu:36,63-100), and which one it
keeps decides the PO obliquity test and the nudge of the reflected ray
(src/cuda/poKernels.cu:91, src/cuda/rtKernels.cu:147-150).  The scene stores each
triangle's rank in the reference's walk for such meshes (tie_order.cpp, checked
against the reference's builder on the CPU by test_tie_order_cpu.py).  Checked here:

* FP64 mode against the reference's own USE_DOUBLE GPU build on the same rays
  (baseline/), where every third triangle of an icosphere is also present reversed;
* the first-hit raster keeps the same triangles as the walk, bit for bit, on that
  mesh (mixed precision).
"""
import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu


def _twin_mesh(seed=3):
    v, t = M.icosphere(3, 1.0)
    rev = t[::3][:, [0, 2, 1]]
    allt = np.concatenate([t, rev])
    return v, allt[np.random.default_rng(seed).permutation(len(allt))]


def test_fp64_matches_reference_double_build_with_coincident_faces():
    ref_gpu = pytest.importorskip("baseline.ref_gpu")
    if not ref_gpu.available(64):
        pytest.skip(f"{ref_gpu.lib_path(64)} not built")
    v, t = _twin_mesh()
    fr, n, G, mb = [3e9, 7e9], 200, 2.2, 3
    th, ph = (40.0, 140.0, 3), (0.0, 315.0, 8)
    r64 = ref_gpu.sweep(v, t, fr, [n] * len(fr), G, mb, 1.0, th, ph, bits=64)
    job = sbr.JobSpec(r64["theta"], r64["phi"], fr, n, n, G, mb, 1.0)
    with sbr.Scene(v, t, device=0) as sc:
        e64 = sbr.run(sc, job, precision=sbr.PREC_FP64).sigma_m2.reshape(-1, len(fr))
    ref = r64["sigma"].T
    ok = ref > 1e-10
    rel = np.abs(e64 - ref)[ok] / ref[ok]
    print(f"coincident faces: FP64 vs the reference's USE_DOUBLE build, max rel sigma diff {rel.max():.3e} "
          f"({ok.sum()} samples)")
    assert rel.max() <= 1e-8


def test_raster_keeps_the_walk_triangles_with_coincident_faces():
    v, t = _twin_mesh()
    job = sbr.JobSpec(np.full(6, 70.0), np.linspace(0.0, 300.0, 6), [5e9, 9e9], 160, 160, 2.2, 3, 1.0)
    with sbr.Scene(v, t, device=0) as sc:
        out = {}
        for fh in (sbr.FIRST_HIT_RASTER, sbr.FIRST_HIT_TRAVERSE):
            r = sbr.run(sc, job, precision=sbr.PREC_MIXED, first_hit=fh)
            out[fh] = (r.field.copy(), r.stats.copy())
    assert np.array_equal(out[sbr.FIRST_HIT_RASTER][0], out[sbr.FIRST_HIT_TRAVERSE][0])
    assert np.array_equal(out[sbr.FIRST_HIT_RASTER][1], out[sbr.FIRST_HIT_TRAVERSE][1])
