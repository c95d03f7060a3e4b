"""The first-hit tile raster (SBR_FIRST_HIT_RASTER, mixed precision) on the benchmark
meshes: the triangles are binned to the trace's 4x8 ray tiles, each tile's list is
tested with the trace's own watertight triangle test, and tiles with more triangles
than the cap walk the tree.  The closest hit is the nearest t, then the lowest
triangle slot, in both the raster and the walk, so the sweep's fields and counters
must equal the walking sweep's bit for bit:

* the seeded 2,148,800-triangle aircraft, 8 azimuths, 8 frequencies (the lane-owned
  epilogue) on the 12,222^2 grid of 18 GHz, 5 bounces, default cap and cap 1 / 8 /
  1024; an FP32 plan asked for the raster walks (the reference's Moller-Trumbore
  test is not watertight);
* the 199,808-triangle SH-displaced ellipsoid at its benchmark size (668^2 rays,
  4 bounces, 121 azimuths), with a graph-captured plan executed twice;
* plans made before sbr_scene_update_vertices: the binning runs at every execution,
  so a stretched mesh is binned as it is now;
* SBR_FIRST_HIT_AUTO (the default) rasterises a mixed-precision plan that launches at
  least 8 rays per triangle per angle and walks otherwise (sbr_plan_info.first_hit).
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


def _same(a, b):
    assert np.array_equal(a.stats, b.stats)
    assert np.array_equal(a.field, b.field)


def test_aircraft_raster_equals_walk():
    v, t = M.aircraft(seed=1)
    G = 2.0 * M.bounding_radius(v)
    n = M.rays_for(18e9, G)
    job = sbr.JobSpec(np.full(8, 90.0), np.linspace(0.0, 315.0, 8), list(np.geomspace(1e9, 18e9, 8)), n, n, G, 5)
    with sbr.Scene(v, t) as sc:
        walk = sbr.run(sc, job, first_hit=sbr.FIRST_HIT_TRAVERSE)
        for cap in (0, 1, 8, 1024):
            _same(sbr.run(sc, job, first_hit=sbr.FIRST_HIT_RASTER, tile_cap=cap), walk)
        _same(sbr.run(sc, job, precision=sbr.PREC_FP32, first_hit=sbr.FIRST_HIT_RASTER),
              sbr.run(sc, job, precision=sbr.PREC_FP32, first_hit=sbr.FIRST_HIT_TRAVERSE))


def test_ellipsoid_raster_equals_walk_graph():
    v, t = M.ellipsoid_sh()
    job = sbr.JobSpec(np.full(121, 90.0), np.linspace(-30.0, 30.0, 121), [5e9], 668, 668, 4.0, 4)
    with sbr.Scene(v, t) as sc:
        walk = sbr.run(sc, job)
        pl = sbr.Plan(sc, [job], use_graph=True, first_hit=sbr.FIRST_HIT_RASTER)
        for _ in range(2):
            pl.execute()
            _same(pl.results(), walk)
        pl.close()


def test_raster_after_vertex_update():
    """A mesh stretched by 1.3 after the plans were made (both keep their launcher
    tables): the raster plan bins the stretched mesh."""
    v, t = M.ellipsoid_sh()
    v = np.asarray(v, np.float32)
    job = sbr.JobSpec(np.full(5, 90.0), np.linspace(-30.0, 30.0, 5), [5e9], 668, 668, 4.0, 4)
    rng = np.random.default_rng(5)
    with sbr.Scene(v, t) as sc:
        pr = sbr.Plan(sc, [job], first_hit=sbr.FIRST_HIT_RASTER)
        pw = sbr.Plan(sc, [job], first_hit=sbr.FIRST_HIT_TRAVERSE)
        sc.update_vertices((v * np.float32(1.3) + rng.normal(0, 2e-3, v.shape)).astype(np.float32))
        pr.execute()
        pw.execute()
        _same(pr.results(), pw.results())
        pr.close()
        pw.close()


def test_auto_first_hit_choice():
    dense_v, dense_t = M.box(1.0)  # 12 triangles, thousands of rays per angle
    sparse_v, sparse_t = M.icosphere(3, 1.0)  # 1,280 triangles, 1,024 rays per angle
    job_dense = sbr.JobSpec([90.0, 60.0], [0.0, 30.0], [3e9], 64, 64, 2.0, 3)
    job_sparse = sbr.JobSpec([90.0, 60.0], [0.0, 30.0], [3e9], 32, 32, 2.2, 3)
    with sbr.Scene(dense_v, dense_t) as sd, sbr.Scene(sparse_v, sparse_t) as ss:
        for sc, job, want in ((sd, job_dense, sbr.FIRST_HIT_RASTER), (ss, job_sparse, sbr.FIRST_HIT_TRAVERSE)):
            pl = sbr.Plan(sc, [job])
            assert pl.info["first_hit"] == want
            pl.execute()
            _same(pl.results(), sbr.run(sc, job, first_hit=sbr.FIRST_HIT_TRAVERSE))
            pl.close()
        pl = sbr.Plan(sd, [job_dense], precision=sbr.PREC_FP32)
        assert pl.info["first_hit"] == sbr.FIRST_HIT_TRAVERSE  # the raster is mixed precision only
        pl.close()
