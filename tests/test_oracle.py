"""CPU tests of the oracle itself: it must reproduce the reference's own outputs
before it is trusted as the checker of the GPU path."""
import json
import os

import numpy as np
import pytest

from oracle import mie
from sagittasbr_b200 import meshes as M

HERE = os.path.dirname(os.path.abspath(__file__))


def _cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.cases()


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_fp64_reproduces_reference_golden(oracle, golden, name):
    """FP64 restatement vs the reference's per-ray routine (oracle/_ref, FP64 build):
    identical hit counts and path lengths per ray, identical fields."""
    v, t, th, ph, fr, nx, ny, G, mb, R = CASES[name]
    out = oracle.sweep(v, t, th, ph, fr, nx, ny, G, mb, R, precision=64, accel="tree", records=True)
    np.testing.assert_array_equal(out.rays["count"], golden[f"{name}/count"].astype(np.int32))
    np.testing.assert_array_equal(out.rays["dist"], golden[f"{name}/dist"])
    np.testing.assert_allclose(out.field, golden[f"{name}/field"], rtol=1e-13, atol=0)


@pytest.mark.parametrize("name", sorted(CASES))
def test_brute_force_matches_tree_walk(oracle, name):
    """Brute force (index order) and the reference tree walk give the same fields
    up to rays flagged ambiguous (exact ties at shared edges)."""
    v, t, th, ph, fr, nx, ny, G, mb, R = CASES[name]
    tree = oracle.sweep(v, t, th, ph, fr, nx, ny, G, mb, R, accel="tree", records=True)
    brute = oracle.sweep(v, t, th, ph, fr, nx, ny, G, mb, R, accel="brute", records=True)
    amb = brute.rays["amb"] != 0
    same = ~amb
    np.testing.assert_array_equal(tree.rays["count"][same], brute.rays["count"][same])
    np.testing.assert_array_equal(tree.rays["tri"][same], brute.rays["tri"][same])
    k = 2 * np.pi * np.asarray(fr) / 299792458.0
    scale = k * (G * G / (nx * ny)) / (4 * np.pi)
    bound = (2 * amb.sum(axis=(1, 2))[:, None] * 2 * scale[None, :] * max(1.0, R) ** mb) + 1e-12
    assert np.all(np.abs(tree.field - brute.field) <= bound)


def test_oracle_matches_reference_live(oracle):
    """When oracle/_ref is built (reference tree present at build time): identical
    SAH trees and bit-identical per-ray records on a fresh case."""
    if not oracle.ref_available(64):
        pytest.skip("oracle/_ref not built")
    v, t = M.icosphere(3, 1.3)
    b1, l1, _ = oracle.build_tree(v, t)
    b2, l2, _ = oracle.build_tree(v, t, source="ref")
    np.testing.assert_array_equal(b1, b2)
    np.testing.assert_array_equal(l1, l2)
    th, ph = [90.0, 37.0], [12.0, 250.0]
    a = oracle.sweep(v, t, th, ph, [2e9], 20, 20, 2.6, 4, records=True)
    r = oracle.ref_sweep(v, t, th, ph, [2e9], 20, 20, 2.6, 4, kind=64, records=True)
    for f in ("count", "dist", "normal", "lastdir"):
        np.testing.assert_array_equal(a.rays[f], r.rays[f])
    np.testing.assert_array_equal(a.field, r.field)


def test_oracle_fp32_tracks_fp64(oracle):
    v, t = M.icosphere(3, 1.0)
    th, ph = np.full(4, 90.0), np.array([3.0, 40.0, 77.0, 130.0])
    a = oracle.sweep(v, t, th, ph, [3e9], 48, 48, 2.0, 3, precision=64)
    b = oracle.sweep(v, t, th, ph, [3e9], 48, 48, 2.0, 3, precision=32)
    assert np.max(np.abs(a.dbsm - b.dbsm)) < 0.1


def test_mie_restatement_matches_reference_function():
    d = json.load(open(os.path.join(HERE, "golden", "mie_ref.json")))
    got = np.array([mie.normalized_rcs(x) for x in d["x"]])
    np.testing.assert_allclose(got, d["normalized_rcs"], rtol=1e-12)
    # headline value at r = 1 m, 1 GHz
    assert abs(mie.sphere_rcs(1.0, 1e9) - 3.02705) < 1e-5


def test_plate_normal_incidence_matches_po_formula(oracle):
    """sigma = 4 pi A_lit^2 / lambda^2 for the rays that hit a flat plate head-on."""
    v, t = M.plate(1.0, 2)
    nx = ny = 40
    G = 1.5
    out = oracle.sweep(v, t, [0.0], [0.0], [5e9], nx, ny, G, 2, records=True)
    lit = (out.rays["count"][0] > 0).sum() * (G * G / (nx * ny))
    lam = 299792458.0 / 5e9
    np.testing.assert_allclose(out.sigma[0, 0], 4 * np.pi * lit ** 2 / lam ** 2, rtol=1e-9)


def test_edge_cases(oracle):
    v, t = M.box(1.0)
    # no bounces allowed -> no field
    out = oracle.sweep(v, t, [30.0], [20.0], [1e9], 8, 8, 2.0, 0)
    assert out.field[0, 0] == 0 and out.counts["queries"][0] == 0
    # a plate seen exactly edge-on is never hit (|det| < 1e-6)
    pv, pt = M.plate(1.0, 1)
    out = oracle.sweep(pv, pt, [90.0], [0.0], [1e9], 16, 16, 2.0, 3)
    assert out.field[0, 0] == 0 and out.counts["hit_rays"][0] == 0
    # single ray grid
    out = oracle.sweep(v, t, [0.0], [0.0], [1e9], 1, 1, 2.0, 3, records=True)
    assert out.rays["count"][0, 0, 0] == 1
    # bad index is rejected
    with pytest.raises(RuntimeError):
        oracle.sweep(v, np.array([[0, 1, 99]]), [0.0], [0.0], [1e9], 2, 2, 2.0, 1)


def test_frame_is_orthogonal_and_matches_reference_layout(oracle):
    for th, ph in [(90, 0), (0, 0), (45, 30), (90, 90), (120, 250)]:
        f = oracle.frame(th, ph, 2.0)
        d, u, v = f["dir"], f["u"], f["v"]
        assert abs(np.dot(d, u)) < 1e-12 and abs(np.dot(d, v)) < 1e-12 and abs(np.dot(u, v)) < 1e-12
        np.testing.assert_allclose([np.linalg.norm(u), np.linalg.norm(v)], [2.0, 2.0], rtol=1e-12)
        np.testing.assert_allclose(f["llc"] + 0.5 * u + 0.5 * v, 20.0 * d, atol=1e-12)


# ------------------------------------------------------------- polarised oracle
# The polarised mode has no reference counterpart; its oracle is pinned to the
# scalar oracle where the two must agree (single bounce) and to closed-form
# physical-optics results where they differ (dihedral and trihedral returns).
C0 = 299792458.0


def test_pol_single_bounce_equals_scalar(oracle):
    """Plate and sphere (single-bounce returns): HH == VV == the scalar field."""
    for (v, t), th, ph, f, n, G in ((M.plate(1.0, 4), [0.0, 10.0, 20.0], [0.0, 30.0, 60.0], 3e9, 100, 1.5),
                                    (M.icosphere(3), [90.0, 90.0], [0.0, 37.0], 1e9, 67, 2.0)):
        s = oracle.sweep(v, t, th, ph, [f], n, n, G, 3).field[:, 0]
        p = oracle.sweep_pol(v, t, th, ph, [f], n, n, G, 3)[:, 0, :]
        tol = 1e-9 * np.abs(s).max()
        assert np.all(np.abs(p[:, 0] - s) <= tol) and np.all(np.abs(p[:, 1] - s) <= tol)


def test_pol_dihedral_broadside(oracle):
    """90-degree dihedral, fold axis along z, seen at broadside (theta 90, phi 45):
    double-bounce returns with HH = -VV and sigma = 8 pi a^2 b^2 / lambda^2
    times cos^2(45 deg) (the ray-tube weighting cos(theta) of the exit term)."""
    v, t = M.dihedral(1.0, 8)
    f = 3e9
    p = oracle.sweep_pol(v, t, [90.0], [45.0], [f], 120, 120, 2.0, 3)[0, 0]
    ratio = p[0] / p[1]
    assert abs(ratio + 1.0) < 2e-3, ratio
    lam = C0 / f
    want = 10 * np.log10(8 * np.pi / lam ** 2 * 0.5)
    got = 10 * np.log10(4 * np.pi * np.abs(p) ** 2)
    assert np.all(np.abs(got - want) < 0.3), (got, want)


def test_pol_trihedral_boresight(oracle):
    """Square trihedral at boresight: triple-bounce returns add in phase with the
    physical exit path, HH = VV, sigma = 12 pi a^4 / lambda^2 times cos^2 = 1/3;
    the scalar reference term (phase 2 k L) decoheres them."""
    v, t = M.trihedral(1.0, 10)
    f = 3e9
    th0 = np.degrees(np.arccos(1 / np.sqrt(3)))
    p = oracle.sweep_pol(v, t, [th0], [45.0], [f], 120, 120, np.sqrt(3), 3)[0, 0]
    s = oracle.sweep(v, t, [th0], [45.0], [f], 120, 120, np.sqrt(3), 3).field[0, 0]
    assert abs(p[0] / p[1] - 1.0) < 2e-3
    lam = C0 / f
    want = 10 * np.log10(12 * np.pi / lam ** 2 / 3)
    got = 10 * np.log10(4 * np.pi * np.abs(p) ** 2)
    assert np.all(np.abs(got - want) < 0.3), (got, want)
    assert 10 * np.log10(4 * np.pi * abs(s) ** 2) < want - 30.0
