"""GPU checks of multi-scene plans (sbr_plan_create_multi): jobs over different
meshes in one persistent launch give the fields of separate single-scene runs (the
fixed-point sums do not depend on which warp adds what): to 1e-12 when the plan's
accumulator layout is each job's own, and within the FP32 partial sums of the
mixed lane-owned layout (below 1e-5) when the plan's widest job selects it for
jobs whose own runs sum per lane in FP64."""
import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def _batch():
    meshes = [M.icosphere(3, 0.7), M.trihedral(0.8, 6), M.box(1.0), M.plate_cluster(4, 3, 0.4, 1.0, seed=3)]
    jobs = [sbr.JobSpec(np.full(20, 90.0), np.linspace(0, 350, 20), [2e9, 3e9], 48, 48, 1.6, 3),
            sbr.JobSpec(np.linspace(10, 80, 15), np.full(15, 45.0), [5e9], 64, 64, 1.5, 3),
            sbr.JobSpec([30.0, 60.0], [10.0, 80.0], [1e9], 40, 40, 2.0, 4),
            sbr.JobSpec(np.full(30, 60.0), np.linspace(0, 300, 30), [4e9, 6e9, 8e9], 56, 56, 2.0, 5, 0.9),
            sbr.JobSpec([45.0, 50.0], [20.0, 25.0], [3e9], 48, 48, 1.6, 2)]
    job_scene = [0, 1, 2, 3, 0]
    return meshes, jobs, job_scene


@pytest.mark.parametrize("prec,pol,mode", [(sbr.PREC_MIXED, sbr.POL_SCALAR, sbr.MODE_BATCHED),
                                           (sbr.PREC_FP32, sbr.POL_SCALAR, sbr.MODE_BATCHED),
                                           (sbr.PREC_FP64, sbr.POL_SCALAR, sbr.MODE_BATCHED),
                                           (sbr.PREC_MIXED, sbr.POL_HHVV, sbr.MODE_BATCHED),
                                           (sbr.PREC_MIXED, sbr.POL_SCALAR, sbr.MODE_PER_ANGLE)])
def test_multi_scene_plan_matches_separate_runs(prec, pol, mode):
    meshes, jobs, job_scene = _batch()
    scenes = [sbr.Scene(v, t) for v, t in meshes]
    try:
        pl = sbr.Plan(scenes, jobs, mode=mode, precision=prec, polarization=pol, job_scene=job_scene)
        pl.execute()
        got = pl.results()
        pl.close()
        want = [sbr.run(scenes[s], j, mode=mode, precision=prec, polarization=pol) for j, s in zip(jobs, job_scene)]
        want_f = np.concatenate([w.field for w in want])
        # the same sums, up to the order of FP64 additions inside a warp when the plan's
        # widest job selects another accumulator layout than a job's own run; the
        # mixed lane-owned layout (more than 4 channels: the HH + VV plan) also sums
        # each 4x8 ray block in FP32 first
        wide = prec == sbr.PREC_MIXED and pol == sbr.POL_HHVV
        rtol, atol = (1e-5, 1e-6) if wide else (1e-12, 1e-13)
        np.testing.assert_allclose(got.field, want_f, rtol=rtol, atol=atol * np.abs(want_f).max())
        assert np.array_equal(got.stats, np.concatenate([w.stats for w in want]))
    finally:
        for s in scenes:
            s.close()


def test_multi_scene_plan_graph_and_repeat():
    meshes, jobs, job_scene = _batch()
    scenes = [sbr.Scene(v, t) for v, t in meshes]
    try:
        pl = sbr.Plan(scenes, jobs, use_graph=True, job_scene=job_scene)
        pl.execute()
        a = pl.results()
        pl.execute()
        b = pl.results()
        pl.close()
        assert np.array_equal(a.field, b.field)
        assert a.field.size == sum(j.n_angles * j.n_freqs for j in jobs)
    finally:
        for s in scenes:
            s.close()


def test_multi_scene_errors():
    meshes, jobs, job_scene = _batch()
    scenes = [sbr.Scene(v, t) for v, t in meshes[:2]]
    try:
        with pytest.raises(sbr.SbrError):
            sbr.Plan(scenes, jobs[:2], job_scene=[0, 2])   # index out of range
        with pytest.raises(ValueError):
            sbr.Plan(scenes, jobs[:2], job_scene=[0])      # one index per job
    finally:
        for s in scenes:
            s.close()


def test_blocks_per_item_and_autotune_keep_the_fields():
    """Work-item size and persistent grid change only how the rays are dealt out:
    fields agree to the FP64 summation order, stats exactly; the autotuner picks
    one of its candidates and reports it."""
    v, t = M.trihedral(1.0, 10)
    job = sbr.JobSpec(np.linspace(20, 70, 12), np.linspace(10, 80, 12), [5e9, 7e9], 96, 96, 1.8, 3)
    with sbr.Scene(v, t) as sc:
        base = sbr.run(sc, job)
        for kw in ({"blocks_per_item": 1}, {"blocks_per_item": 16, "ctas_per_sm": 6}, {"autotune": True}):
            pl = sbr.Plan(sc, [job], **kw)
            pl.execute()
            r = pl.results()
            info = pl.info
            pl.close()
            np.testing.assert_allclose(r.field, base.field, rtol=1e-12, atol=1e-13 * np.abs(base.field).max())
            assert np.array_equal(r.stats, base.stats)
            if kw.get("autotune"):
                assert info["blocks_per_item"] in (0, 1, 2, 4, 8, 16) and info["ctas_per_sm"] in (0, 6)
            else:
                assert info["blocks_per_item"] == kw["blocks_per_item"]
