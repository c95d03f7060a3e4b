"""FP64 reference gradient of the scalar PO field sweep along frozen hit paths.

Test infrastructure only (the GPU adjoint, sbr_adjoint, is checked against it; the
product never imports it).  The reference has no gradient; this restates the
quantity the adjoint differentiates, independently of its reverse sweep:

  * hit sequences from the FP64 oracle's own trace (oracle_sweep with records, the
    reference SAH tree walk of src/cuda/rtKernels.cu:63-158);
  * per ray, the path through that frozen triangle sequence re-evaluated in FP64
    from the vertices (ray-plane distance t = ((a - o).N) / (d.N), hit point, unit
    normal unit(e1 x e2), reflection d - 2 (d.n) n, nudge p + 1e-4 n,
    src/cuda/rtKernels.cu:126-158) and its exit term
    k A / (4 pi) * 2 cos R^n * j exp(j 2 k L)   (src/cuda/poKernels.cu:81-109),
    with the cos > 0 gate held fixed;
  * d(term)/d(vertex coordinate) by central differences of that FP64 path
    (step `delta`, 1e-6 m: truncation O(delta^2), rounding of the 40 m launcher
    path about 1e-12 rad of phase, so about 1e-8 relative).
Only rays whose frozen path touches a triangle of the vertex change, so only those
are re-evaluated.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O

C0 = 299792458.0


def _path_terms(P, tri_idx, seq, count, o0, d0, k, area, R):
    """Complex field terms [rays, freqs] of rays with frozen triangle sequences
    seq [rays, B] (caller triangle ids) and hit counts, launched at o0 along d0."""
    o, d = o0.copy(), d0.copy()
    L = np.zeros(o.shape[0])
    nl = np.zeros_like(o)
    dl = np.zeros_like(o)
    for b in range(seq.shape[1]):
        live = count > b
        if not live.any():
            break
        t_id = np.where(live, seq[:, b], 0)
        a, bb, c = P[tri_idx[t_id, 0]], P[tri_idx[t_id, 1]], P[tri_idx[t_id, 2]]
        N = np.cross(bb - a, c - a)
        t = ((a - o) * N).sum(1) / (d * N).sum(1)
        n = N / np.linalg.norm(N, axis=1)[:, None]
        p = o + t[:, None] * d
        dn = (d * n).sum(1)
        dnew = d - 2.0 * dn[:, None] * n
        dnew = dnew / np.linalg.norm(dnew, axis=1)[:, None]
        onew = p + 1e-4 * n
        L = np.where(live, L + t, L)
        nl = np.where(live[:, None], n, nl)
        dl = np.where(live[:, None], d, dl)
        o = np.where(live[:, None], onew, o)
        d = np.where(live[:, None], dnew, d)
    cos = -(nl * dl).sum(1)
    mag = (k[None, :] * area / (4.0 * np.pi)) * (2.0 * cos * np.power(R, count))[:, None]
    ph = 2.0 * k[None, :] * L[:, None]
    return mag * (-np.sin(ph) + 1j * np.cos(ph))


def frozen_path_gradient(verts, tris, theta_deg, phi_deg, freqs_hz, nx, ny, grid_size, max_bounces, cot,
                         vertex_ids, reflection_const=1.0, model_scale=1.0, delta=1e-6, threads=0):
    """dLoss/d(vertex position) for the listed vertices, [len(vertex_ids), 3], where
    dLoss = sum_s Re(conj(cot_s) dS_s) over the samples (angle-major, then
    frequency) of the FP64 sweep; also returns the oracle's fields [angles, freqs]."""
    v32 = np.asarray(verts, dtype=np.float32).reshape(-1, 3)
    T = np.asarray(tris, dtype=np.int64).reshape(-1, 3)
    th = np.asarray(theta_deg, dtype=np.float64).ravel()
    ph = np.asarray(phi_deg, dtype=np.float64).ravel()
    fr = np.asarray(freqs_hz, dtype=np.float64).ravel()
    out = O.sweep(v32, T.astype(np.uint32), th, ph, fr, nx, ny, grid_size, max_bounces, reflection_const,
                  precision=64, accel="tree", threads=threads, records=True, model_scale=model_scale)
    rec = out.rays.reshape(th.size, -1)
    g = np.asarray(cot, dtype=np.complex128).reshape(th.size, fr.size)
    k = 2.0 * np.pi * fr / C0
    area = grid_size * grid_size / (nx * ny)
    P0 = v32.astype(np.float64) * model_scale
    cnt_all = rec["count"]
    seq_all = rec["tri"][:, :, :max(1, max_bounces)]
    # gate of the base path: rays whose exit cos <= 0 add nothing (held fixed)
    cos_all = -(rec["normal"] * rec["lastdir"]).sum(-1)
    keep_all = (cnt_all > 0) & (cos_all > 0)
    incident = [[] for _ in range(P0.shape[0])]
    for ti, (a, b, c) in enumerate(T):
        incident[a].append(ti)
        incident[b].append(ti)
        incident[c].append(ti)
    frames = [O.frame(a, b, grid_size) for a, b in zip(th, ph)]
    jj, ii = np.divmod(np.arange(nx * ny), nx)
    u, vv = (ii + 0.5) / nx, (jj + 0.5) / ny
    grad = np.zeros((len(vertex_ids), 3))
    for row, vid in enumerate(vertex_ids):
        tri_set = np.asarray(incident[int(vid)], dtype=np.int64)
        for a in range(th.size):
            touch = keep_all[a] & np.isin(seq_all[a], tri_set).any(axis=1)
            if not touch.any():
                continue
            f = frames[a]
            o0 = f["llc"][None, :] + u[touch, None] * f["u"][None, :] + vv[touch, None] * f["v"][None, :]
            d0 = np.broadcast_to(-f["dir"], o0.shape).copy()
            seq, cnt = seq_all[a][touch], cnt_all[a][touch]
            for c in range(3):
                Pp, Pm = P0.copy(), P0.copy()
                Pp[vid, c] += delta
                Pm[vid, c] -= delta
                dS = (_path_terms(Pp, T, seq, cnt, o0, d0, k, area, reflection_const).sum(0)
                      - _path_terms(Pm, T, seq, cnt, o0, d0, k, area, reflection_const).sum(0)) / (2.0 * delta)
                grad[row, c] += float(np.real(np.conj(g[a]) * dS).sum())
    # the caller's coordinates are scaled by model_scale before tracing
    return grad * model_scale, out.field
