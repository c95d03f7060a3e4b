"""GPU checks of sbr_scene_update_vertices (new vertices, BVH refitted on the GPU):
a refitted scene must trace exactly like a scene built from scratch on the same
vertices -- same bounds, same closest hits, bitwise the same triangle data --
because a BVH only prunes and the triangle tests decide every hit.  Rays the FP64
brute-force oracle flags as ambiguous (shared edges, thresholds, ties), where the
traversal order of the two trees may pick another triangle, are left out, and the
fields may differ by at most those rays' terms."""
import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu

C0 = 299792458.0


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


@pytest.mark.parametrize("deform", ["small", "large"])
def test_refit_traces_like_a_fresh_build(oracle, deform):
    v0, t = M.ellipsoid_sh(n_theta=24, n_phi=48)
    rng = np.random.default_rng(3)
    if deform == "small":
        v1 = (v0 + rng.normal(0.0, 2e-3, v0.shape)).astype(np.float32)
    else:
        v1 = (1.7 * v0[:, [1, 2, 0]] + np.array([0.3, -0.2, 0.1]) + rng.normal(0.0, 0.02, v0.shape)).astype(np.float32)
    job = sbr.JobSpec([90.0, 60.0, 20.0], [0.0, 45.0, 200.0], [3e9, 5e9], 72, 72, 6.0, 4)
    o = oracle.sweep(v1, t, job.theta_deg, job.phi_deg, job.freqs_hz, 72, 72, 6.0, 4, accel="brute",
                     records=True, amb_edge=1e-6, amb_t=1e-6)
    ok = o.rays["amb"] == 0
    assert ok.mean() > 0.9
    with sbr.Scene(v0, t, want_fp64=True) as a, sbr.Scene(v1, t, want_fp64=True) as b:
        a.update_vertices(v1)
        ia, ib = a.info(), b.info()
        assert ia["aabb_lo"] == ib["aabb_lo"] and ia["aabb_hi"] == ib["aabb_hi"]
        for prec in (sbr.PREC_FP64, sbr.PREC_MIXED, sbr.PREC_FP32):
            ra = sbr.trace_records(a, job, precision=prec)
            rb = sbr.trace_records(b, job, precision=prec)
            for key in ("count", "tri", "dist", "normal", "lastdir"):
                assert np.array_equal(ra[key][ok], rb[key][ok]), (prec, key)
            fa = sbr.run(a, job, precision=prec).field.reshape(3, 2)
            fb = sbr.run(b, job, precision=prec).field.reshape(3, 2)
            k = 2 * np.pi * np.array([3e9, 5e9]) / C0
            scale = k * (6.0 * 6.0 / (72 * 72)) / (4 * np.pi)
            namb = (~ok).sum(axis=(1, 2))
            bound = scale[None, :] * 4.0 * namb[:, None] + 1e-12 * np.abs(fb).max()
            assert np.all(np.abs(fa - fb) <= bound), prec
        # the adjoint follows the new vertices too
        cot = np.ones(6, complex)
        ga, fa_ = sbr.adjoint(a, job, cot, precision=sbr.PREC_FP64)
        gb, fb_ = sbr.adjoint(b, job, cot, precision=sbr.PREC_FP64)
        assert np.linalg.norm(ga - gb) <= 1e-6 * np.linalg.norm(gb) + 4.0 * (~ok).sum() * np.abs(gb).max()


def test_refit_errors():
    v, t = M.box(1.0)
    with sbr.Scene(v, t) as sc:
        with pytest.raises(sbr.SbrError) as e:
            sc.update_vertices(v[:-1])
        assert e.value.status == 1
        bad = v.copy()
        bad[0, 0] = np.nan
        with pytest.raises(sbr.SbrError) as e:
            sc.update_vertices(bad)
        assert e.value.status == 4
        # a failed update leaves the scene as it was
        r = sbr.run(sc, sbr.JobSpec([30.0], [20.0], [1e9], 16, 16, 2.0, 3))
        assert r.stats[0, 1] > 0
