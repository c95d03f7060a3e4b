"""GPU parity: libsbr (sm_100a, through the C ABI) against the CPU oracle and the
reference's own golden outputs.

Tolerances (per (angle, frequency) complex field S):
    |S_gpu - S_ref| <= scale_k * (4 * n_amb * Rmax + eps * sum_r amp_r)
where scale_k = k A_ray / (4 pi), n_amb = rays the FP64 brute-force oracle flags
as ambiguous (a decision within 1e-6 m / 1e-6 relative of flipping: shared
edges, |det| at the 1e-6 threshold, ties in t, t at tMin), each of which can
change the sum by at most 2 * max|term|, and amp_r = 2 cos(theta) R^n is the
magnitude of ray r's term.  eps is the per-ray phase/amplitude error of the
precision mode: 1e-9 (FP64), 1e-4 (mixed: FP32 traversal, FP32-pair phase), 3e-3
(FP32: the reference FP32 build's arithmetic, FP32 phase at 10 G).
Hit sequences must be identical for every ray the oracle does not flag.
"""
import os

import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
C0 = 299792458.0
EPS = {sbr.PREC_FP64: 1e-9, sbr.PREC_MIXED: 1e-4, sbr.PREC_FP32: 3e-3}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def _cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.cases()


CASES = _cases()


def amp_sum(records, R):
    """sum over rays of 2 cos(theta) R^n per angle, from oracle records."""
    cnt = records["count"]
    c = -(records["normal"] * records["lastdir"]).sum(axis=-1)
    a = np.where((cnt > 0) & (c > 0), 2.0 * c * np.power(R, cnt), 0.0)
    return a.sum(axis=(1, 2))


def field_bound(oracle_out, freqs, G, nx, ny, R, max_bounces, prec):
    k = 2 * np.pi * np.asarray(freqs) / C0
    scale = k * (G * G / (nx * ny)) / (4 * np.pi)
    namb = (oracle_out.rays["amb"] != 0).sum(axis=(1, 2))
    rmax = max(1.0, abs(R)) ** max_bounces
    return scale[None, :] * (4.0 * namb[:, None] * rmax + EPS[prec] * amp_sum(oracle_out.rays, R)[:, None]) + 1e-300


def oracle_brute(oracle, case):
    v, t, th, ph, fr, nx, ny, G, mb, R = case
    return oracle.sweep(v, t, th, ph, fr, nx, ny, G, mb, R, accel="brute", records=True, amb_edge=1e-6, amb_t=1e-6)


@pytest.fixture(scope="module")
def brute(oracle):
    return {name: oracle_brute(oracle, CASES[name]) for name in CASES}


@pytest.mark.parametrize("prec", [sbr.PREC_FP64, sbr.PREC_MIXED, sbr.PREC_FP32])
@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_fields(golden, brute, name, prec):
    v, t, th, ph, fr, nx, ny, G, mb, R = CASES[name]
    with sbr.Scene(v, t) as sc:
        res = sbr.run(sc, sbr.JobSpec(th, ph, fr, nx, ny, G, mb, R), precision=prec)
    got = res.field.reshape(len(th), len(fr))
    ref = golden[f"{name}/field"]
    bound = field_bound(brute[name], fr, G, nx, ny, R, mb, prec)
    err = np.abs(got - ref)
    assert np.all(err <= bound), (name, prec, err.max(), (err / bound).max())


@pytest.mark.parametrize("prec", [sbr.PREC_FP64, sbr.PREC_MIXED])
@pytest.mark.parametrize("name", sorted(CASES))
def test_hit_sequences(brute, name, prec):
    """Identical triangle-hit sequences and counts for every unambiguous ray."""
    v, t, th, ph, fr, nx, ny, G, mb, R = CASES[name]
    with sbr.Scene(v, t) as sc:
        rec = sbr.trace_records(sc, sbr.JobSpec(th, ph, fr, nx, ny, G, mb, R), precision=prec)
    o = brute[name].rays
    ok = o["amb"] == 0
    assert ok.mean() > 0.9
    np.testing.assert_array_equal(rec["count"][ok], o["count"][ok])
    np.testing.assert_array_equal(rec["tri"][ok], o["tri"][ok])
    hit = ok & (o["count"] > 0)
    tol = 1e-9 if prec == sbr.PREC_FP64 else 2e-5
    assert np.all(np.abs(rec["dist"][hit] - o["dist"][hit]) <= tol * np.maximum(1.0, o["dist"][hit]))
    np.testing.assert_allclose(rec["normal"][hit], o["normal"][hit], atol=1e-5)


@pytest.mark.parametrize("name", sorted(CASES))
def test_first_hit_raster_matches_walk(golden, brute, name):
    """The first-hit tile raster (mixed precision) gives exactly the walk's records on
    every ray (the closest hit is the nearest t, then the tie order, in both) and
    bitwise the walk's fields, whether the tiles test their lists (cap 1024), walk
    (cap 1) or both (the default cap); FP32 plans asked for the raster walk."""
    v, t, th, ph, fr, nx, ny, G, mb, R = CASES[name]
    job = sbr.JobSpec(th, ph, fr, nx, ny, G, mb, R)
    o = brute[name].rays
    ok = o["amb"] == 0
    with sbr.Scene(v, t) as sc:
        for prec in (sbr.PREC_MIXED, sbr.PREC_FP32):
            walk = sbr.trace_records(sc, job, precision=prec, first_hit=sbr.FIRST_HIT_TRAVERSE)
            for cap in (0, 1, 1024):
                rec = sbr.trace_records(sc, job, precision=prec, first_hit=sbr.FIRST_HIT_RASTER, tile_cap=cap)
                for f in ("count", "flags", "tri", "dist", "normal", "lastdir"):
                    np.testing.assert_array_equal(rec[f], walk[f], err_msg=f"{f}, tile_cap {cap}")
            if prec == sbr.PREC_MIXED:
                np.testing.assert_array_equal(walk["tri"][ok], o["tri"][ok])
            res = sbr.run(sc, job, precision=prec, first_hit=sbr.FIRST_HIT_RASTER)
            res_w = sbr.run(sc, job, precision=prec, first_hit=sbr.FIRST_HIT_TRAVERSE)
            assert np.array_equal(res.field, res_w.field)
            assert np.array_equal(res.stats, res_w.stats)
            bound = field_bound(brute[name], fr, G, nx, ny, R, mb, prec)
            assert np.all(np.abs(res.field.reshape(len(th), len(fr)) - golden[f"{name}/field"]) <= bound)


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_hit_counts(golden, brute, name):
    """GPU FP64 hit counts and paths against the reference's own per-ray output."""
    v, t, th, ph, fr, nx, ny, G, mb, R = CASES[name]
    with sbr.Scene(v, t) as sc:
        rec = sbr.trace_records(sc, sbr.JobSpec(th, ph, fr, nx, ny, G, mb, R), precision=sbr.PREC_FP64)
    ok = brute[name].rays["amb"] == 0
    np.testing.assert_array_equal(rec["count"][ok], golden[f"{name}/count"][ok])
    np.testing.assert_allclose(rec["dist"][ok], golden[f"{name}/dist"][ok], rtol=1e-12, atol=1e-12)


def test_batched_equals_per_angle_and_is_deterministic():
    v, t = M.icosphere(3, 1.0)
    th = np.full(24, 90.0)
    ph = np.linspace(0, 345, 24)
    job = sbr.JobSpec(th, ph, [2e9, 3e9], 64, 64, 2.0, 3)
    with sbr.Scene(v, t) as sc:
        a = sbr.run(sc, job, mode=sbr.MODE_BATCHED)
        b = sbr.run(sc, job, mode=sbr.MODE_BATCHED)
        c = sbr.run(sc, job, mode=sbr.MODE_PER_ANGLE)
    assert np.array_equal(a.field, b.field)  # bitwise reproducible
    np.testing.assert_allclose(a.field, c.field, rtol=1e-12, atol=1e-14 * np.abs(a.field).max())
    np.testing.assert_array_equal(a.stats, c.stats)


def test_many_frequencies_one_trace(oracle):
    """40 frequencies share one trace (lane-per-frequency epilogue) and match the
    oracle, which re-evaluates the PO term per frequency on the same rays."""
    v, t = M.trihedral(1.0, 6)
    th, ph = [54.7356, 40.0, 70.0], [45.0, 30.0, 60.0]
    fr = np.geomspace(2e9, 9e9, 40)
    G, nx, mb = 2.0 * M.bounding_radius(v), 48, 3
    with sbr.Scene(v, t) as sc:
        res = sbr.run(sc, sbr.JobSpec(th, ph, fr, nx, nx, G, mb), precision=sbr.PREC_FP64)
    o = oracle.sweep(v, t, th, ph, fr, nx, nx, G, mb, accel="brute", records=True)
    bound = field_bound(o, fr, G, nx, nx, 1.0, mb, sbr.PREC_FP64)
    assert np.all(np.abs(res.field.reshape(3, 40) - o.field) <= bound)


def test_several_jobs_in_one_plan_match_separate_runs():
    v, t = M.box(1.0)
    j1 = sbr.JobSpec([30.0, 60.0], [10.0, 80.0], [1e9], 40, 40, 2.0, 4)
    j2 = sbr.JobSpec([45.0], [45.0], [3e9, 4e9], 70, 50, 2.5, 2, 0.8)
    with sbr.Scene(v, t) as sc:
        both = sbr.run(sc, [j1, j2])
        a = sbr.run(sc, j1)
        b = sbr.run(sc, j2)
    np.testing.assert_allclose(both.field, np.concatenate([a.field, b.field]), rtol=1e-13)


def test_edge_cases(oracle):
    v, t = M.box(1.0)
    with sbr.Scene(v, t) as sc:
        # no bounces: nothing is traced
        r = sbr.run(sc, sbr.JobSpec([30.0], [20.0], [1e9], 8, 8, 2.0, 0))
        assert r.field[0] == 0 and r.stats.sum() == 0
        # odd grids, 1x1 grid, the up=(1,0,0) branch (|dir.y| > 0.99), poles
        for (nx, ny, th, ph) in [(17, 33, 35.0, 10.0), (1, 1, 0.0, 0.0), (9, 5, 90.0, 90.0), (12, 12, 180.0, 0.0),
                                 (20, 20, 90.0, 270.0)]:
            r = sbr.run(sc, sbr.JobSpec([th], [ph], [2e9], nx, ny, 2.0, 3), precision=sbr.PREC_FP64)
            o = oracle.sweep(v, t, [th], [ph], [2e9], nx, ny, 2.0, 3, accel="brute", records=True)
            assert np.all(np.abs(r.field - o.field.ravel()) <= field_bound(o, [2e9], 2.0, nx, ny, 1.0, 3,
                                                                             sbr.PREC_FP64).ravel())
            assert int(r.stats[0, 1]) == int(o.counts["hit_rays"][0])
        # a launcher much wider than the body: the clipped aperture gives the same field
        r = sbr.run(sc, sbr.JobSpec([50.0], [20.0], [1e9], 400, 400, 20.0, 3), precision=sbr.PREC_FP64)
        o = oracle.sweep(v, t, [50.0], [20.0], [1e9], 400, 400, 20.0, 3)
        np.testing.assert_allclose(r.field, o.field.ravel(), rtol=1e-9)
        assert r.stats[0, 0] < 400 * 400 // 10
    # edge-on plate: never hit
    pv, pt = M.plate(1.0, 1)
    with sbr.Scene(pv, pt) as sc:
        r = sbr.run(sc, sbr.JobSpec([90.0], [0.0], [1e9], 16, 16, 2.0, 3))
        assert r.field[0] == 0 and r.stats[0, 1] == 0


def test_error_statuses():
    v, t = M.box(1.0)
    with sbr.Scene(v, t) as sc:
        for bad in [sbr.JobSpec([0.0], [0.0], [1e9], 0, 4, 2.0, 3),
                    sbr.JobSpec([0.0], [0.0], [-1.0], 4, 4, 2.0, 3),
                    sbr.JobSpec([0.0], [0.0], [1e9], 4, 4, -2.0, 3),
                    sbr.JobSpec([np.nan], [0.0], [1e9], 4, 4, 2.0, 3)]:
            with pytest.raises(sbr.SbrError):
                sbr.run(sc, bad)
        with pytest.raises(sbr.SbrError) as e:
            sbr.run(sc, sbr.JobSpec([0.0], [0.0], np.linspace(1e9, 2e9, 129), 4, 4, 2.0, 3))
        assert e.value.status == 5
        with pytest.raises(sbr.SbrError) as e:
            sbr.run(sc, sbr.JobSpec([0.0], [0.0], [1e9], 70000, 70000, 2.0, 3))
        assert e.value.status == 5
        # cancel flag observed by the kernel -> SBR_ERR_CANCELLED, scene still usable
        sc.cancel()
        with pytest.raises(sbr.SbrError) as e:
            sbr.run(sc, sbr.JobSpec(np.zeros(64), np.linspace(0, 90, 64), [1e9], 64, 64, 2.0, 3))
        assert e.value.status == 11
        sc.reset_cancel()
        r = sbr.run(sc, sbr.JobSpec([0.0], [0.0], [1e9], 8, 8, 2.0, 3))
        assert r.stats[0, 1] > 0


def test_sphere_sweep_against_oracle_and_mie(oracle):
    """Icosphere level 5 (20480 tris), 1 GHz, 67x67 rays, 3 bounces, 360 azimuths."""
    from oracle import mie
    v, t = M.icosphere(5, 1.0)
    th = np.full(360, 90.0)
    ph = np.arange(360.0)
    n = M.rays_for(1e9, 2.0)
    assert n == 67
    with sbr.Scene(v, t) as sc:
        res = {p: sbr.run(sc, sbr.JobSpec(th, ph, [1e9], n, n, 2.0, 3), precision=p)
               for p in (sbr.PREC_MIXED, sbr.PREC_FP64, sbr.PREC_FP32)}
    o = oracle.sweep(v, t, th, ph, [1e9], n, n, 2.0, 3, precision=64)
    ref_db = o.dbsm.ravel()
    # At phi = 0, sin(phi) = 0 exactly: the middle ray row lies in the mesh's y = 0
    # symmetry plane with d.y = -0, and the reference slab test evaluates 0 * inf =
    # NaN for boxes with a face at y = 0 (src/cuda/rtKernels.cu:47-55), dropping
    # them; its tree walk then misses hits that the closest-hit definition (brute
    # force over every triangle) finds.  That angle is compared with brute force.
    ob = oracle.sweep(v, t, [90.0], [0.0], [1e9], n, n, 2.0, 3, precision=64, accel="brute")
    assert abs(ob.dbsm[0, 0] - ref_db[0]) > 0.1  # the reference walk's loss is real
    ref_db[0] = ob.dbsm[0, 0]
    for p, r in res.items():
        assert np.max(np.abs(r.rcs_dbsm - ref_db)) <= 0.1, (p, np.max(np.abs(r.rcs_dbsm - ref_db)))
    sigma_mie = mie.sphere_rcs(1.0, 1e9)
    assert abs(np.mean(res[sbr.PREC_MIXED].sigma_m2) / sigma_mie - 1) < 0.1


def test_trihedral_full_resolution_against_oracle(oracle):
    """Square trihedral, 60k triangles, 10 GHz, 578^2 rays, 3 bounces, at the
    boresight and off it.  Compared with the FP64 oracle walking the reference
    tree: |dS| <= 1e-3 * sum_r |term_r| (precision and edge flips together).
    The reference's phase is 2 k times the summed path from the launcher
    (src/cuda/poKernels.cu:95), not the retro-reflected round trip, so the
    triple-bounce rays do not add in phase at the boresight as a physical
    corner reflector's would; the oracle is the only pin."""
    v, t = M.trihedral(1.0, 100)
    G = 2.0 * M.bounding_radius(v)
    n = M.rays_for(1e10, G)
    assert n == 578
    th, ph = [54.7356103172, 20.0], [45.0, 70.0]
    with sbr.Scene(v, t) as sc:
        r = sbr.run(sc, sbr.JobSpec(th, ph, [1e10], n, n, G, 3))
        recs = sbr.trace_records(sc, sbr.JobSpec(th, ph, [1e10], n, n, G, 3))
    o = oracle.sweep(v, t, th, ph, [1e10], n, n, G, 3, precision=64, accel="tree")
    k = 2 * np.pi * 1e10 / C0
    scale = k * (G * G / (n * n)) / (4 * np.pi)
    c = -(recs["normal"] * recs["lastdir"]).sum(axis=-1)
    absum = scale * np.where((recs["count"] > 0) & (c > 0), 2 * c, 0).sum(axis=(1, 2))
    assert np.all(np.abs(r.field - o.field.ravel()) <= 1e-3 * absum)
    assert np.all(r.stats[:, 1] == o.counts["hit_rays"]) or \
        np.all(np.abs(r.stats[:, 1].astype(float) - o.counts["hit_rays"]) <= 1e-4 * n * n)
    assert r.stats[0, 2] > 2.5 * r.stats[0, 1]  # boresight: mostly triple bounces
