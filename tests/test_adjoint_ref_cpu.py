"""CPU pin of the FP64 reference gradient (oracle/adjoint_ref.py) used to check the
GPU adjoint: on a small SH-displaced ellipsoid its frozen-path derivative equals
central finite differences of the FP64 oracle sweep (full re-trace, h = 1e-5 m in
FP32 vertex coordinates) on every component whose +-h runs keep every ray's hit
sequence.  Loss = mean sigma over the samples."""
import numpy as np

from sagittasbr_b200 import meshes as M


def test_frozen_path_gradient_matches_oracle_finite_differences(oracle):
    from oracle.adjoint_ref import frozen_path_gradient
    v, t = M.ellipsoid_sh(n_theta=24, n_phi=48)
    v = np.asarray(v, np.float32)
    th, ph, fr, n, G, mb = [90.0, 60.0], [0.0, 45.0], [3e9, 4e9], 64, 4.0, 3
    base = oracle.sweep(v, t, th, ph, fr, n, n, G, mb, precision=64, records=True)
    S = base.field.ravel()
    cot = 8.0 * np.pi * S / S.size
    hit_tris = np.unique(base.rays["tri"][base.rays["tri"] >= 0])
    lit = np.unique(np.asarray(t)[hit_tris].ravel())
    vids = np.random.default_rng(1).choice(lit, 5, replace=False)
    g, field = frozen_path_gradient(v, t, th, ph, fr, n, n, G, mb, cot, vids)
    np.testing.assert_array_equal(field, base.field)
    valid = 0
    for r, vid in enumerate(vids):
        for c in range(3):
            vp, vm = v.copy(), v.copy()
            vp[vid, c] = np.float32(v[vid, c] + 1e-5)
            vm[vid, c] = np.float32(v[vid, c] - 1e-5)
            op = oracle.sweep(vp, t, th, ph, fr, n, n, G, mb, precision=64, records=True)
            om = oracle.sweep(vm, t, th, ph, fr, n, n, G, mb, precision=64, records=True)
            if not (np.array_equal(op.rays["tri"], base.rays["tri"]) and
                    np.array_equal(om.rays["tri"], base.rays["tri"])):
                continue
            valid += 1
            fd = (op.sigma.mean() - om.sigma.mean()) / (float(vp[vid, c]) - float(vm[vid, c]))
            assert abs(g[r, c] - fd) <= 1e-4 * abs(fd) + 1e-9 * np.abs(g).max(), (vid, c, g[r, c], fd)
    assert valid >= 10
