"""The adjoint at the differentiable-shape benchmark size, through the C ABI.

SH-displaced ellipsoid 2/1/0.5 m (199,808 triangles, seeded 32-mode displacement),
5 GHz, G = 4 m, 668^2 rays, 4 bounces, five of the 121 azimuths over -30..30 deg,
loss = mean sigma (m^2) over those samples.  sbr_adjoint (FP64) is checked on 64
seeded vertices with a non-zero gradient:

* against the FP64 reference gradient of oracle/adjoint_ref.py -- the frozen-path
  derivative of the oracle's own FP64 trace, by central differences of the FP64
  path algebra -- on every component;
* against central finite differences of the GPU FP64 sweep (h = 1e-5 m, the FP32
  step actually stored; the scene refitted for each +-h run) on every component
  whose +-h runs keep every ray's hit sequence: the per-angle ray / hit / bounce /
  query counts must be unchanged and the rays whose base path touches the vertex's
  two-ring of triangles must hit the same triangles (sbr_trace_ray_list).  The
  share of masked components is reported in the failure message.
Tolerances: reference gradient |g - g_ref| <= 1e-5 |g_ref| + 1e-7 max|g|;
finite differences |g - fd| <= 1e-3 |fd| + 1e-6 max|g| (the adjoint target).
The differentiated term is src/cuda/poKernels.cu:81-109 along src/cuda/rtKernels.cu:126-158.
"""
import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu

PHI = np.array([-30.0, -15.0, 0.0, 15.0, 30.0])
F, G, MB = 5e9, 4.0, 4


@pytest.fixture(scope="module")
def setup():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    v, t = M.ellipsoid_sh()
    v = np.asarray(v, np.float32)
    assert t.shape[0] == 199808
    n = M.rays_for(F, G)
    assert n == 668
    job = sbr.JobSpec(np.full(PHI.size, 90.0), PHI, [F], n, n, G, MB)
    sc = sbr.Scene(v, t, want_fp64=True)
    base = sbr.run(sc, job, precision=sbr.PREC_FP64)
    cot = 8.0 * np.pi * base.field / base.field.size
    g, gf = sbr.adjoint(sc, job, cot, precision=sbr.PREC_FP64)
    lit = np.flatnonzero(np.abs(g).sum(axis=1) > 0)
    assert lit.size >= 64
    picks = np.random.default_rng(64).choice(lit, 64, replace=False)
    yield dict(v=v, t=t, n=n, job=job, sc=sc, base=base, cot=cot, g=g, picks=picks)
    sc.close()


def test_adjoint_matches_fp64_reference_gradient(setup):
    from oracle.adjoint_ref import frozen_path_gradient
    s = setup
    g_ref, field = frozen_path_gradient(s["v"], s["t"], s["job"].theta_deg, PHI, [F], s["n"], s["n"], G, MB,
                                        s["cot"], s["picks"])
    # the oracle's FP64 sweep is the engine's FP64 sweep
    np.testing.assert_allclose(s["base"].field, field.ravel(), rtol=1e-9, atol=1e-12 * np.abs(field).max())
    g = s["g"][s["picks"]]
    tol = 1e-5 * np.abs(g_ref) + 1e-7 * np.abs(s["g"]).max()
    bad = np.argwhere(np.abs(g - g_ref) > tol)
    assert bad.size == 0, [(int(s["picks"][r]), int(c), g[r, c], g_ref[r, c]) for r, c in bad[:10]]


def test_adjoint_matches_finite_differences_at_config_size(setup):
    s = setup
    v, t, sc, job = s["v"], s["t"], s["sc"], s["job"]
    rec0 = sbr.trace_records(sc, job, precision=sbr.PREC_FP64).reshape(PHI.size, -1)
    tri0 = rec0["tri"][:, :, :MB]
    stats0 = s["base"].stats
    incident = {}
    for ti, tri in enumerate(t):
        for q in tri:
            incident.setdefault(int(q), []).append(ti)
    gmax = np.abs(s["g"]).max()
    valid, masked, bad = 0, 0, []
    h = 1e-5
    for vid in s["picks"]:
        ring1 = set(incident[int(vid)])
        ring2 = np.array(sorted({tt for tri in ring1 for q in t[tri] for tt in incident[int(q)]}))
        touch = np.argwhere(np.isin(tri0, ring2).any(axis=2))  # (angle, ray) pairs
        rays = np.stack([touch[:, 0], touch[:, 1] % s["n"], touch[:, 1] // s["n"]], axis=1)
        want = tri0[touch[:, 0], touch[:, 1]]
        for c in range(3):
            vp, vm = v.copy(), v.copy()
            vp[vid, c] = np.float32(v[vid, c] + h)
            vm[vid, c] = np.float32(v[vid, c] - h)
            loss, same = [], True
            for vv in (vp, vm):
                sc.update_vertices(vv)
                r = sbr.run(sc, job, precision=sbr.PREC_FP64)
                loss.append(float(r.sigma_m2.mean()))
                same &= np.array_equal(r.stats, stats0)
                if rays.shape[0]:
                    same &= np.array_equal(sbr.trace_ray_list(sc, job, rays, precision=sbr.PREC_FP64)["tri"][:, :MB],
                                           want)
            if not same:
                masked += 1
                continue
            valid += 1
            fd = (loss[0] - loss[1]) / (float(vp[vid, c]) - float(vm[vid, c]))
            if abs(s["g"][vid, c] - fd) > 1e-3 * abs(fd) + 1e-6 * gmax:
                bad.append((int(vid), c, float(s["g"][vid, c]), fd))
    sc.update_vertices(v)
    total = 3 * len(s["picks"])
    assert valid >= total // 2, f"{masked} of {total} components masked by hit-sequence changes"
    assert not bad, (f"{len(bad)} of {valid} components off ({masked} of {total} masked)", bad[:10])
