"""The GPU SAH build (sbr_build_opts.gpu_build) against the host build: the same
binary tree (node count, depth, bounds) and 4-wide layout, and the same fields
(leaf triangle order may differ, which only reorders exact ties)."""
import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu


def _duplicates():
    """40 copies of one triangle (identical centroids: the median-split fallback)
    beside a small icosphere."""
    v, t = M.icosphere(2, 1.0)
    tri = np.array([[0.0, 0.0, 0.0], [0.3, 0.0, 0.0], [0.0, 0.3, 0.0]], np.float32) + 2.0
    vd = np.concatenate([v, tri]).astype(np.float32)
    base = v.shape[0]
    td = np.concatenate([t, np.tile(np.array([[base, base + 1, base + 2]]), (40, 1))]).astype(np.uint32)
    return vd, td


MESHES = {
    "one_triangle": lambda: (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.uint32)),
    "icosphere4": lambda: M.icosphere(4, 1.0),
    "trihedral": lambda: M.trihedral(1.0, 40),
    "plates": lambda: M.plate_cluster(24, 12, seed=5),
    "duplicates": _duplicates,
    "ellipsoid_sh": lambda: M.ellipsoid_sh(),
}


@pytest.mark.parametrize("name", list(MESHES))
def test_gpu_build_matches_host_build(name):
    v, t = MESHES[name]()
    with sbr.Scene(v, t, want_fp64=True) as host, sbr.Scene(v, t, want_fp64=True, gpu_build=True) as gpu:
        a, b = host.info(), gpu.info()
        for k in ("n_nodes_bin", "n_nodes_gpu", "bvh_depth", "aabb_lo", "aabb_hi", "device_bytes"):
            assert a[k] == b[k], (k, a[k], b[k])
        G = 2.0 * M.bounding_radius(v) + 0.1
        job = sbr.JobSpec([90.0, 60.0, 30.0, 5.0], [10.0, 45.0, 200.0, 300.0], [3e9], 96, 96, G, 4)
        for prec in (sbr.PREC_FP64, sbr.PREC_MIXED):
            ra, rb = sbr.run(host, job, precision=prec), sbr.run(gpu, job, precision=prec)
            np.testing.assert_array_equal(ra.stats, rb.stats)
            scale = max(np.abs(ra.field).max(), 1e-30)
            assert np.abs(ra.field - rb.field).max() <= 1e-9 * scale, name


def test_gpu_build_is_faster_on_a_large_mesh():
    v, t = M.ellipsoid_sh(n_theta=400, n_phi=800)  # 638k triangles
    with sbr.Scene(v, t) as host, sbr.Scene(v, t, gpu_build=True) as gpu:
        a, b = host.info(), gpu.info()
        print(f"{t.shape[0]} triangles: host SAH {a['sah_ms']:.1f} ms, GPU SAH {b['sah_ms']:.1f} ms")
        assert a["n_nodes_bin"] == b["n_nodes_bin"] and a["bvh_depth"] == b["bvh_depth"]
