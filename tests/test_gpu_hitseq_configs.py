"""Hit-sequence parity on the benchmark configurations, through the C ABI.

The golden-mesh parity tests use small grids; these take the meshes, ray grids and
bounce limits of the benchmark workloads: the level-5 icosphere at 1 GHz (67^2 rays,
3 bounces, every ray of four azimuths), and seeded samples of the rays launched on
the 60,000-triangle trihedral (578^2 grid, 3 bounces), the 199,808-triangle
SH-displaced ellipsoid (668^2, 4 bounces) and the 2,148,800-triangle aircraft
(12,222^2 grid of 18 GHz, 5 bounces).  sbr_trace_ray_list traces only the sampled
rays with the sweep's own walk; the FP64 brute-force oracle traces the same rays over
every triangle and flags the ones whose decision lies within 1e-6 (m, relative) of
flipping (src/cuda/rtKernels.cu:10-44,105-158).  Every unflagged ray must hit the same
triangles in the same order, with the same count, in FP64 and in mixed precision.
"""
import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def _compare(rec, o, prec):
    ok = o["amb"] == 0
    assert ok.mean() > 0.9
    np.testing.assert_array_equal(rec["count"][ok], o["count"][ok])
    np.testing.assert_array_equal(rec["tri"][ok], o["tri"][ok])
    hit = ok & (o["count"] > 0)
    assert hit.sum() > 0.2 * ok.size
    tol = 1e-9 if prec == sbr.PREC_FP64 else 2e-5
    assert np.all(np.abs(rec["dist"][hit] - o["dist"][hit]) <= tol * np.maximum(1.0, o["dist"][hit]))
    np.testing.assert_allclose(rec["normal"][hit], o["normal"][hit], atol=1e-5)


@pytest.mark.parametrize("prec", [sbr.PREC_FP64, sbr.PREC_MIXED, sbr.PREC_FP32])
def test_ray_list_equals_full_records(prec):
    """sbr_trace_ray_list gives exactly the records sbr_trace_records gives for the
    same rays."""
    v, t = M.icosphere(3, 1.0)
    th, ph = np.array([90.0, 45.0, 10.0]), np.array([0.0, 123.0, 300.0])
    job = sbr.JobSpec(th, ph, [3e9], 40, 40, 2.0, 4)
    rng = np.random.default_rng(2)
    rays = np.stack([rng.integers(0, 3, 500), rng.integers(0, 40, 500), rng.integers(0, 40, 500)], axis=1)
    with sbr.Scene(v, t) as sc:
        full = sbr.trace_records(sc, job, precision=prec)
        lst = sbr.trace_ray_list(sc, job, rays, precision=prec)
    ref = full[rays[:, 0], rays[:, 2], rays[:, 1]]
    launched = ref["flags"] == 1
    for f in ("count", "dist", "normal", "lastdir", "tri"):
        np.testing.assert_array_equal(lst[f][launched], ref[f][launched])
    # rays outside the clipped aperture are not launched by the sweep and hit nothing
    assert np.all(lst["count"][~launched] == 0)


def test_ray_list_rejects_rays_outside_the_job():
    v, t = M.icosphere(2, 1.0)
    job = sbr.JobSpec([90.0], [0.0], [1e9], 16, 16, 2.0, 2)
    with sbr.Scene(v, t) as sc:
        for bad in ([1, 0, 0], [0, 16, 0], [0, 0, -1]):
            with pytest.raises(sbr.SbrError):
                sbr.trace_ray_list(sc, job, np.array([bad]))


@pytest.mark.parametrize("prec", [sbr.PREC_FP64, sbr.PREC_MIXED])
def test_sphere_config_every_ray(oracle, prec):
    """Icosphere level 5 (20,480 triangles), 1 GHz, G = 2 m, 67^2 rays, 3 bounces:
    every ray of four azimuths."""
    v, t = M.icosphere(5, 1.0)
    ph = np.array([0.0, 37.0, 90.0, 211.0])
    th = np.full(4, 90.0)
    n = M.rays_for(1e9, 2.0)
    assert n == 67
    with sbr.Scene(v, t) as sc:
        rec = sbr.trace_records(sc, sbr.JobSpec(th, ph, [1e9], n, n, 2.0, 3), precision=prec)
    o = oracle.sweep(v, t, th, ph, [1e9], n, n, 2.0, 3, accel="brute", records=True)
    launched = rec["flags"] == 1
    # every ray the oracle sees hitting was launched (aperture clipping loses nothing)
    assert np.all(launched[o.rays["count"] > 0])
    _compare(rec, o.rays, prec)


def _sampled(oracle, v, t, th, ph, f, G, mb, per_angle, prec):
    n = M.rays_for(f, G)
    rays = oracle.sample_rays(v, th, ph, n, n, G, per_angle, seed=17)
    with sbr.Scene(v, t) as sc:
        rec = sbr.trace_ray_list(sc, sbr.JobSpec(th, ph, [f], n, n, G, mb), rays, precision=prec)
    o, _ = oracle.trace_rays(v, t, th, ph, rays, n, n, G, mb, accel="brute")
    _compare(rec, o, prec)


@pytest.mark.parametrize("prec", [sbr.PREC_FP64, sbr.PREC_MIXED])
def test_trihedral_config_sampled_rays(oracle, prec):
    v, t = M.trihedral(1.0, 100)
    G = 2.0 * M.bounding_radius(v)
    assert M.rays_for(1e10, G) == 578
    _sampled(oracle, v, t, np.array([54.7356, 30.0, 80.0, 5.0]), np.array([45.0, 10.0, 60.0, 85.0]), 1e10, G, 3,
             2000, prec)


@pytest.mark.parametrize("prec", [sbr.PREC_FP64, sbr.PREC_MIXED])
def test_ellipsoid_config_sampled_rays(oracle, prec):
    v, t = M.ellipsoid_sh()
    assert M.rays_for(5e9, 4.0) == 668
    _sampled(oracle, v, t, np.full(4, 90.0), np.array([-30.0, -7.5, 12.5, 30.0]), 5e9, 4.0, 4, 2000, prec)


@pytest.mark.parametrize("prec", [sbr.PREC_FP64, sbr.PREC_MIXED])
def test_aircraft_config_sampled_rays(oracle, prec):
    v, t = M.aircraft(seed=1)
    G = 2.0 * M.bounding_radius(v)
    assert M.rays_for(18e9, G) == 12222
    _sampled(oracle, v, t, np.full(3, 90.0), np.array([0.0, 30.0, 90.0]), 18e9, G, 5, 300, prec)
