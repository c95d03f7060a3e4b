"""The stated error of mixed-precision results against FP64 (sbr_error_bound).

For every sample of a mixed-precision sweep the engine can state its error against
the FP64 sweep of the same job (the reference's USE_DOUBLE arithmetic): exact for
the rays near a decision (re-traced in FP64), a probabilistic rounding bound for
the rest.  The statement must hold -- |field - field_FP64| and |dBsm - dBsm_FP64|
at or below the stated values on every sample, unfiltered -- on the benchmark's
sphere (icosphere level 5, 1 GHz, 67^2 rays, 3 bounces) and trihedral (60,000
triangles, 578^2 rays, 3 bounces, theta and phi over 0..90) configurations, and it
must be informative where the answer is well conditioned (the sphere; the
trihedral within 30 dB of each frequency's peak).
The row it annotates is src/app/sweep.cu:540-544 (rcs_results.csv).
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


def _check(v, t, job):
    with sbr.Scene(v, t, want_fp64=True) as sc:
        a = sbr.run(sc, job, precision=sbr.PREC_MIXED)
        b = sbr.run(sc, job, precision=sbr.PREC_FP64)
        ef, ed = sbr.error_bound(sc, job, a)
    df = np.abs(a.field - b.field)
    ddb = np.abs(a.rcs_dbsm - b.rcs_dbsm)
    assert np.all(df <= ef), (np.argmax(df / ef), (df / ef).max())
    # the statement is not vacuous: it is below |field| on most samples
    assert np.mean(ef < np.abs(a.field)) > 0.5
    assert np.all(ddb <= ed + 1e-9), (np.argmax(ddb - ed), ddb.max(), ed[np.argmax(ddb - ed)])
    return ddb, ed


def test_bound_holds_on_the_sphere_config():
    v, t = M.icosphere(5, 1.0)
    job = sbr.JobSpec(np.full(36, 90.0), np.arange(0.0, 360.0, 10.0), [1e9], 67, 67, 2.0, 3)
    ddb, ed = _check(v, t, job)
    assert np.median(ed) < 0.01, np.median(ed)


def test_bound_holds_on_the_trihedral_config():
    v, t = M.trihedral(1.0, 100)
    G = 2.0 * M.bounding_radius(v)
    g = np.linspace(0.0, 90.0, 8)
    th, ph = np.meshgrid(g, g, indexing="ij")
    job = sbr.JobSpec(th.ravel(), ph.ravel(), [8e9, 1e10], M.rays_for(1e10, G), M.rays_for(1e10, G), G, 3)
    ddb, ed = _check(v, t, job)
    with sbr.Scene(v, t) as sc:
        db = sbr.run(sc, job).rcs_dbsm.reshape(-1, 2)
    near = (db > db.max(axis=0)[None, :] - 30.0).ravel()
    assert np.median(ed[near]) < 0.1, np.median(ed[near])


def test_bound_rejects_other_precisions():
    v, t = M.icosphere(2, 1.0)
    job = sbr.JobSpec([90.0], [0.0], [1e9], 16, 16, 2.0, 2)
    with sbr.Scene(v, t) as sc:
        r = sbr.run(sc, job)
        f = np.ascontiguousarray(np.stack([r.field.real, r.field.imag], axis=1).ravel())
        o = sbr._opts(sbr.MODE_BATCHED, sbr.PREC_FP64)
        jc = sbr._jobs_c([job])
        assert sbr.lib().sbr_error_bound(sc.handle, jc, 1, sbr.C.byref(o), sbr._p(f), None, None) == 14
