"""GPU parity of the polarised mode (SBR_POL_HHVV) against the FP64 polarised
oracle (oracle.sweep_pol), whose own closed-form checks are in test_oracle.py.

Tolerance per (angle, frequency, polarisation) field S:
    |S_gpu - S_oracle| <= scale_k * (4 * n_amb * Rmax + eps * 2 * n_hit * Rmax)
with n_amb the rays the FP64 brute-force oracle flags as ambiguous (each can move
the sum by at most twice the largest term), n_hit the rays with at least one hit
(each term is at most 2 R^n in amplitude), eps 1e-9 for FP64 and 5e-4 for mixed
precision (FP32 hit points enter the exit path: about 1e-7 relative times k |p|).
"""
import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu

C0 = 299792458.0
EPS = {sbr.PREC_FP64: 1e-9, sbr.PREC_MIXED: 5e-4}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def _case(name):
    th0 = float(np.degrees(np.arccos(1 / np.sqrt(3))))
    if name == "dihedral":
        v, t = M.dihedral(1.0, 8)
        return v, t, [90.0, 90.0, 80.0, 60.0], [45.0, 40.0, 45.0, 20.0], 2.0, 96, 3
    if name == "trihedral":
        v, t = M.trihedral(1.0, 10)
        return v, t, [th0, 50.0, 30.0], [45.0, 40.0, 70.0], float(np.sqrt(3)), 96, 3
    if name == "sphere":
        v, t = M.icosphere(3)
        return v, t, [90.0, 90.0, 45.0], [0.0, 37.0, 200.0], 2.0, 67, 3
    v, t = M.box(1.0)
    return v, t, [30.0, 50.0, 0.0], [10.0, 20.0, 0.0], 2.0, 64, 4


def _bound(oracle, v, t, th, ph, fr, n, G, mb, prec):
    o = oracle.sweep(v, t, th, ph, [fr[0]], n, n, G, mb, accel="brute", records=True, amb_edge=1e-6, amb_t=1e-6)
    namb = (o.rays["amb"] != 0).sum(axis=(1, 2))
    nhit = (o.rays["count"] > 0).sum(axis=(1, 2))
    k = 2 * np.pi * np.asarray(fr) / C0
    scale = k * (G * G / (n * n)) / (4 * np.pi)
    b = scale[None, :] * (4.0 * namb[:, None] + EPS[prec] * 2.0 * nhit[:, None]) + 1e-300
    return b[:, :, None]


@pytest.mark.parametrize("nf", [1, 2, 3, 40])
@pytest.mark.parametrize("prec", [sbr.PREC_FP64, sbr.PREC_MIXED])
@pytest.mark.parametrize("name", ["dihedral", "trihedral", "sphere", "box"])
def test_pol_fields_match_oracle(oracle, name, prec, nf):
    """HH and VV fields, batched, for 1 / 2 / 3 / 40 frequencies per job (2, 4, 6
    and 80 accumulation channels: per-lane and lane-per-channel epilogues)."""
    v, t, th, ph, G, n, mb = _case(name)
    fr = np.geomspace(2e9, 4e9, nf) if nf > 1 else np.array([3e9])
    with sbr.Scene(v, t) as sc:
        res = sbr.run(sc, sbr.JobSpec(th, ph, fr, n, n, G, mb), precision=prec, polarization=sbr.POL_HHVV)
    got = res.field.reshape(len(th), nf, 2)
    want = oracle.sweep_pol(v, t, th, ph, fr, n, n, G, mb, accel="brute")
    bound = _bound(oracle, v, t, th, ph, fr, n, G, mb, prec)
    err = np.abs(got - want)
    assert np.all(err <= bound), (name, prec, nf, err.max(), (err / bound).max())
    np.testing.assert_allclose(res.sigma_m2.reshape(len(th), nf, 2), 4 * np.pi * np.abs(got) ** 2, rtol=1e-12)


def test_pol_per_angle_equals_batched_and_is_deterministic():
    v, t, th, ph, G, n, mb = _case("dihedral")
    job = sbr.JobSpec(th, ph, [2e9, 3e9], n, n, G, mb)
    with sbr.Scene(v, t) as sc:
        a = sbr.run(sc, job, polarization=sbr.POL_HHVV)
        b = sbr.run(sc, job, polarization=sbr.POL_HHVV)
        c = sbr.run(sc, job, mode=sbr.MODE_PER_ANGLE, polarization=sbr.POL_HHVV)
        s = sbr.run(sc, job)
    assert a.field.shape == (len(th) * 2, 2)
    assert np.array_equal(a.field, b.field)
    np.testing.assert_allclose(a.field, c.field, rtol=1e-12, atol=1e-14 * np.abs(a.field).max())
    np.testing.assert_array_equal(a.stats, s.stats)


def test_pol_single_bounce_equals_scalar():
    """A plate at several angles: single-bounce returns give HH == VV == scalar."""
    v, t = M.plate(1.0, 4)
    job = sbr.JobSpec([0.0, 10.0, 20.0], [0.0, 30.0, 60.0], [3e9], 100, 100, 1.5, 3)
    with sbr.Scene(v, t) as sc:
        p = sbr.run(sc, job, precision=sbr.PREC_FP64, polarization=sbr.POL_HHVV)
        s = sbr.run(sc, job, precision=sbr.PREC_FP64)
    tol = 1e-9 * np.abs(s.field).max()
    assert np.all(np.abs(p.field[:, 0] - s.field) <= tol)
    assert np.all(np.abs(p.field[:, 1] - s.field) <= tol)


def test_pol_plan_info_and_errors():
    v, t = M.box(1.0)
    with sbr.Scene(v, t) as sc:
        pl = sbr.Plan(sc, [sbr.JobSpec([10.0], [20.0], [1e9, 2e9], 16, 16, 2.0, 3)], polarization=sbr.POL_HHVV)
        assert pl.info["n_pol"] == 2
        pl.execute()
        r = pl.results()
        assert r.field.shape == (2, 2) and r.rcs_dbsm.shape == (2, 2)
        pl.close()
        with pytest.raises(sbr.SbrError) as e:  # FP32 arithmetic is the reference's scalar path only
            sbr.run(sc, sbr.JobSpec([0.0], [0.0], [1e9], 8, 8, 2.0, 3), precision=sbr.PREC_FP32,
                    polarization=sbr.POL_HHVV)
        assert e.value.status == 14
        with pytest.raises(sbr.SbrError) as e:  # 65 frequencies x 2 polarisations > 128 channels
            sbr.run(sc, sbr.JobSpec([0.0], [0.0], np.linspace(1e9, 2e9, 65), 8, 8, 2.0, 3),
                    polarization=sbr.POL_HHVV)
        assert e.value.status == 5
