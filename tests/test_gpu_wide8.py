"""The opt-in 8-wide BVH (sbr_build_opts.node_width = 8): the mixed-precision
scalar sweep walks 8-wide nodes over the same leaves as the 4-wide tree, so it must
find the same closest hits.  On flat plates (trihedral, where two triangles that
tie at a shared edge have the same normal and hit point) the fields are equal bit
for bit; on the icosphere within the ambiguity bound of the parity tests (a tie at
a shared edge may pick the other triangle).  Other precisions and kernels walk the
4-wide tree of the same scene."""
import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def _both(v, t, job, prec=sbr.PREC_MIXED):
    with sbr.Scene(v, t) as s4, sbr.Scene(v, t, node_width=8) as s8:
        assert s8.info()["device_bytes"] > s4.info()["device_bytes"]
        return sbr.run(s4, job, precision=prec), sbr.run(s8, job, precision=prec)


def test_trihedral_fields_equal_bitwise():
    v, t = M.trihedral(1.0, 30)
    th, ph = np.meshgrid(np.linspace(0, 90, 7), np.linspace(0, 90, 7), indexing="ij")
    job = sbr.JobSpec(th.ravel(), ph.ravel(), [6e9, 1e10], 200, 200, 2.0 * M.bounding_radius(v), 3)
    a, b = _both(v, t, job)
    np.testing.assert_array_equal(a.field, b.field)
    np.testing.assert_array_equal(a.stats, b.stats)


def test_sphere_fields_agree_and_other_precisions_unchanged():
    v, t = M.icosphere(4, 1.0)
    job = sbr.JobSpec(np.full(24, 90.0), np.linspace(0, 345, 24), [2e9, 3e9], 96, 96, 2.0, 3)
    a, b = _both(v, t, job)
    assert np.abs(a.field - b.field).max() <= 1e-3 * np.abs(a.field).max()
    np.testing.assert_array_equal(a.stats[:, :2], b.stats[:, :2])
    for prec in (sbr.PREC_FP64, sbr.PREC_FP32):
        x, y = _both(v, t, job, prec)
        np.testing.assert_array_equal(x.field, y.field)


def test_node_width_validation_and_refit_drops_the_wide_tree():
    v, t = M.icosphere(2, 1.0)
    with pytest.raises(sbr.SbrError):
        sbr.Scene(v, t, node_width=6)
    job = sbr.JobSpec([90.0], [10.0], [1e9], 32, 32, 2.0, 2)
    with sbr.Scene(v, t, node_width=8) as s8, sbr.Scene(v, t) as s4:
        v2 = (np.asarray(v) * 1.01).astype(np.float32)
        s8.update_vertices(v2)
        s4.update_vertices(v2)
        np.testing.assert_array_equal(sbr.run(s8, job).field, sbr.run(s4, job).field)


def test_plan_node_width_and_autotuned_width():
    """A plan walks the scene's widest tree by default, the 4-wide one on request,
    and the autotuner times both widths when the scene holds an 8-wide tree."""
    v, t = M.trihedral(1.0, 20)
    th, ph = np.meshgrid(np.linspace(5, 85, 5), np.linspace(5, 85, 5), indexing="ij")
    job = sbr.JobSpec(th.ravel(), ph.ravel(), [1e10], 160, 160, 2.0 * M.bounding_radius(v), 3)
    with sbr.Scene(v, t, node_width=8) as s8, sbr.Scene(v, t) as s4:
        ref = sbr.run(s4, job).field
        for kw, want in (({}, 8), ({"node_width": 4}, 4), ({"node_width": 8}, 8), ({"autotune": True}, None)):
            pl = sbr.Plan(s8, [job], **kw)
            assert pl.info["node_width"] == (want if want else pl.info["node_width"])
            assert pl.info["node_width"] in (4, 8)
            pl.execute()
            np.testing.assert_array_equal(pl.results().field, ref)
            pl.close()
        assert sbr.Plan(s4, [job]).info["node_width"] == 4
        with pytest.raises(sbr.SbrError):
            sbr.Plan(s4, [job], node_width=8)
