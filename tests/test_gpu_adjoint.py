"""GPU checks of the adjoint (sbr_adjoint): vertex and frequency gradients of the
mean RCS against central finite differences of the FP64 sweep.

Finite differences see the hit / miss and triangle-switch discontinuities that the
frozen-path gradient leaves out, so a component is compared only when the ray hit
sequences of its +h and -h runs equal those of the base run (sbr_trace_records,
FP64); at least half of the sampled components must qualify.  Vertices are stored
in FP32, so the step is the difference of the FP32 coordinates actually used.
Tolerance per component: |grad - fd| <= 1e-3 |fd| + 1e-6 max|grad|.
"""
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


def _loss_and_tri(v, t, job):
    with sbr.Scene(v, t, want_fp64=True) as sc:
        r = sbr.run(sc, job, precision=sbr.PREC_FP64)
        rec = sbr.trace_records(sc, job, precision=sbr.PREC_FP64)
    return float(r.sigma_m2.mean()), rec["tri"].copy()


def _fd_check(v, t, job, n_pick, seed, h=1e-5):
    v = np.asarray(v, np.float32)
    with sbr.Scene(v, t, want_fp64=True) as sc:
        base = sbr.run(sc, job, precision=sbr.PREC_FP64)
        rec0 = sbr.trace_records(sc, job, precision=sbr.PREC_FP64)["tri"]
        cot = 8.0 * np.pi * base.field / base.field.size
        g, _ = sbr.adjoint(sc, job, cot, precision=sbr.PREC_FP64)
    lit = np.flatnonzero(np.abs(g).sum(axis=1) > 0)
    assert lit.size >= n_pick
    rng = np.random.default_rng(seed)
    picks = rng.choice(lit, n_pick, replace=False)
    gmax = np.abs(g).max()
    valid, bad = 0, []
    for vi in picks:
        for c in range(3):
            vp, vm = v.copy(), v.copy()
            vp[vi, c] = np.float32(v[vi, c] + h)
            vm[vi, c] = np.float32(v[vi, c] - h)
            lp, tp = _loss_and_tri(vp, t, job)
            lm, tm = _loss_and_tri(vm, t, job)
            if not (np.array_equal(tp, rec0) and np.array_equal(tm, rec0)):
                continue
            valid += 1
            fd = (lp - lm) / (float(vp[vi, c]) - float(vm[vi, c]))
            if abs(g[vi, c] - fd) > 1e-3 * abs(fd) + 1e-6 * gmax:
                bad.append((int(vi), c, float(g[vi, c]), fd))
    return valid, 3 * n_pick, bad, g


def test_adjoint_vertices_match_finite_differences_ellipsoid():
    """SH-displaced ellipsoid (2208 triangles), 3 angles, 3 bounces."""
    v, t = M.ellipsoid_sh(n_theta=24, n_phi=48)
    job = sbr.JobSpec([90.0, 90.0, 60.0], [0.0, 20.0, 45.0], [3e9], 80, 80, 4.0, 3)
    valid, total, bad, _ = _fd_check(v, t, job, 12, seed=1)
    assert valid >= total // 2, (valid, total)
    assert not bad, bad


def test_adjoint_vertices_match_finite_differences_multibounce():
    """Dihedral and trihedral (two triangles per plate): gradients through
    double and triple reflections."""
    for (v, t), th, ph, G in ((M.dihedral(1.0, 1), [90.0, 80.0], [40.0, 50.0], 2.0),
                              (M.trihedral(1.0, 1), [50.0, 60.0], [40.0, 35.0], float(np.sqrt(3)))):
        job = sbr.JobSpec(th, ph, [3e9], 64, 64, G, 3)
        valid, total, bad, g = _fd_check(v, t, job, min(4, v.shape[0]), seed=2)
        assert valid >= total // 2, (valid, total)
        assert not bad, bad


def test_adjoint_frequency_matches_finite_differences():
    v, t = M.ellipsoid_sh(n_theta=24, n_phi=48)
    th, ph = [90.0, 70.0], [10.0, 30.0]
    f0, df = 3e9, 2e3
    fr = [f0, 4e9]
    job = sbr.JobSpec(th, ph, fr, 80, 80, 4.0, 3)
    with sbr.Scene(v, t, want_fp64=True) as sc:
        base = sbr.run(sc, job, precision=sbr.PREC_FP64)
        w = np.ones(base.field.size) / base.field.size
        _, gf = sbr.adjoint(sc, job, 8.0 * np.pi * w * base.field, precision=sbr.PREC_FP64)
        for k, f in enumerate(fr):
            fp = list(fr)
            fm = list(fr)
            fp[k], fm[k] = f + df, f - df
            lp = sbr.run(sc, sbr.JobSpec(th, ph, fp, 80, 80, 4.0, 3), precision=sbr.PREC_FP64).sigma_m2.mean()
            lm = sbr.run(sc, sbr.JobSpec(th, ph, fm, 80, 80, 4.0, 3), precision=sbr.PREC_FP64).sigma_m2.mean()
            fd = (lp - lm) / (2 * df)
            ad = gf.reshape(len(th), len(fr))[:, k].sum()
            assert abs(ad - fd) <= 1e-3 * abs(fd) + 1e-18, (k, ad, fd)


def test_adjoint_mixed_matches_fp64():
    """Mixed precision re-traces with the FP32 walk and differentiates in FP64:
    the same gradient as the FP64 walk up to the rays whose FP32 hits differ."""
    v, t = M.ellipsoid_sh(n_theta=48, n_phi=96)
    job = sbr.JobSpec([90.0, 80.0], [0.0, 33.0], [5e9, 6e9], 120, 120, 4.0, 4)
    with sbr.Scene(v, t, want_fp64=True) as sc:
        base = sbr.run(sc, job, precision=sbr.PREC_FP64)
        cot = 8.0 * np.pi * base.field / base.field.size
        g64, f64 = sbr.adjoint(sc, job, cot, precision=sbr.PREC_FP64)
        gmx, fmx = sbr.adjoint(sc, job, cot, precision=sbr.PREC_MIXED)
    assert np.linalg.norm(gmx - g64) <= 1e-2 * np.linalg.norm(g64)
    assert np.all(np.abs(fmx - f64) <= 1e-2 * np.abs(f64).max())


def test_torch_autograd_bridge():
    import torch
    from sagittasbr_b200.autograd import rcs
    v, t = M.ellipsoid_sh(n_theta=24, n_phi=48)
    th, ph = np.array([90.0, 60.0]), np.array([0.0, 45.0])
    verts = torch.tensor(v, dtype=torch.float64, requires_grad=True)
    freqs = torch.tensor([3e9, 5e9], dtype=torch.float64, requires_grad=True)
    sigma = rcs(verts, t, th, ph, freqs, 64, 64, 4.0, 3, precision=sbr.PREC_FP64)
    assert sigma.shape == (2, 2)
    loss = (sigma * torch.tensor([[1.0, 2.0], [0.5, 1.0]], dtype=torch.float64)).sum()
    loss.backward()
    with sbr.Scene(v, t, want_fp64=True) as sc:
        job = sbr.JobSpec(th, ph, [3e9, 5e9], 64, 64, 4.0, 3)
        base = sbr.run(sc, job, precision=sbr.PREC_FP64)
        w = np.array([1.0, 2.0, 0.5, 1.0])
        g, gf = sbr.adjoint(sc, job, 8.0 * np.pi * w * base.field, precision=sbr.PREC_FP64)
    np.testing.assert_allclose(sigma.detach().numpy().ravel(), base.sigma_m2, rtol=1e-12)
    np.testing.assert_allclose(verts.grad.numpy(), g, rtol=1e-9, atol=1e-12 * np.abs(g).max())
    np.testing.assert_allclose(freqs.grad.numpy(), gf.reshape(2, 2).sum(axis=0), rtol=1e-9)


def test_adjoint_errors():
    v, t = M.box(1.0)
    with sbr.Scene(v, t) as sc:
        job = sbr.JobSpec([30.0], [10.0], [1e9], 16, 16, 2.0, 17)
        with pytest.raises(sbr.SbrError) as e:
            sbr.adjoint(sc, job, np.zeros(1, complex))
        assert e.value.status == 5
        with pytest.raises(ValueError):
            sbr.adjoint(sc, sbr.JobSpec([30.0], [10.0], [1e9], 16, 16, 2.0, 3), np.zeros(2, complex))
