"""ctypes front-end for the CPU oracle (oracle/sbr_oracle.cpp) and for the
reference's own per-ray routine compiled for the host (oracle/_ref).

Test infrastructure only: imported by tests/, the smoke check and bench.py's
cpu_baseline / reference legs, never by the product package.

References restated by the C++ side are listed in oracle/sbr_oracle.cpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import time
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = {
    64: os.path.join(HERE, "_ref", "libsbrref64.so"),
    32: os.path.join(HERE, "_ref", "libsbrref32.so"),
    "32fast": os.path.join(HERE, "_ref", "libsbrref32_fast.so"),
}
MAX_REC = 16

# Ambiguity flag bits (sbr_oracle.cpp)
AMB_EDGE, AMB_DET, AMB_TIE, AMB_TMIN = 1, 2, 4, 8

ORACLE_RAY = np.dtype(
    [
        ("count", np.int32),
        ("amb", np.int32),
        ("dist", np.float64),
        ("normal", np.float64, 3),
        ("lastdir", np.float64, 3),
        ("tri", np.int32, MAX_REC),
    ],
    align=True,
)
REF_RAY = np.dtype(
    [
        ("count", np.int32),
        ("pad", np.int32),
        ("dist", np.float64),
        ("normal", np.float64, 3),
        ("lastdir", np.float64, 3),
    ],
    align=True,
)
COUNTS = np.dtype(
    [
        ("rays", np.uint64),
        ("hit_rays", np.uint64),
        ("bounces", np.uint64),
        ("queries", np.uint64),
        ("box_tests", np.uint64),
        ("tri_tests", np.uint64),
    ]
)

_P = C.c_void_p
_I64 = C.c_int64
_I32 = C.c_int32
_D = C.c_double


def build(force: bool = False) -> None:
    """Compile the oracle (and oracle/_ref when the reference tree exists)."""
    if force or not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.oracle_sweep.restype = C.c_int
        L.oracle_sweep.argtypes = [
            _P, _I64, _P, _I64, _D,
            _P, _P, _I64, _P, _I64,
            _I32, _I32, _D, _I32, _D,
            _I32, _I32, _I32, _P, _P,
            _P, _P, _D, _D, _D,
        ]
        L.oracle_sweep_pol.restype = C.c_int
        L.oracle_sweep_pol.argtypes = [
            _P, _I64, _P, _I64, _D,
            _P, _P, _I64, _P, _I64,
            _I32, _I32, _D, _I32, _D,
            _I32, _I32, _P, _P,
        ]
        L.oracle_trace_rays.restype = C.c_int
        L.oracle_trace_rays.argtypes = [
            _P, _I64, _P, _I64, _D,
            _P, _P, _I64, _P, _I64,
            _I32, _I32, _D, _I32, _I32,
            _I32, _I32, _P, _P, _D, _D, _D,
        ]
        L.oracle_build_tree.restype = _I64
        L.oracle_build_tree.argtypes = [_P, _I64, _P, _I64, _D, _P, _P, _P]
        L.oracle_frame.restype = None
        L.oracle_frame.argtypes = [_D, _D, _D, _P]
        L.oracle_ray_record_size.restype = C.c_int
        assert L.oracle_ray_record_size() == ORACLE_RAY.itemsize, "oracle_ray layout mismatch"
        _lib = L
    return _lib


def ref_available(kind=64) -> bool:
    return os.path.exists(REF_SO[kind])


def ref_lib(kind=64):
    if kind not in _ref:
        L = C.CDLL(REF_SO[kind])
        L.ref_sweep.restype = C.c_int
        L.ref_sweep.argtypes = [
            _P, _I64, _P, _I64, _D,
            _P, _P, _I64, _P, _I64,
            _I32, _I32, _D, _I32, _D, _I32,
            _P, _P, _P, _P,
        ]
        L.ref_build_tree.restype = _I64
        L.ref_build_tree.argtypes = [_P, _I64, _P, _I64, _D, _P, _P, _P]
        L.ref_real_bytes.restype = C.c_int
        L.ref_scene_create.restype = C.c_void_p
        L.ref_scene_create.argtypes = [_P, _I64, _P, _I64, _D]
        L.ref_scene_destroy.restype = None
        L.ref_scene_destroy.argtypes = [_P]
        L.ref_trace_rows.restype = C.c_int
        L.ref_trace_rows.argtypes = [_P, _P, _P, _I64, _P, _I64, _P, _D, _I32, _D, _I32, _P, _P, _P, _P, _P]
        _ref[kind] = L
    return _ref[kind]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class SweepOut:
    field: np.ndarray  # complex128 [n_angles, n_freqs]
    counts: np.ndarray | None = None  # COUNTS [n_angles]
    rays: np.ndarray | None = None  # per-ray records [n_angles, ny, nx]

    @property
    def sigma(self):
        return 4.0 * np.pi * (self.field.real ** 2 + self.field.imag ** 2)

    @property
    def dbsm(self):
        return 10.0 * np.log10(np.maximum(self.sigma, 1e-10))


def _mesh_args(verts, tris):
    v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tris, dtype=np.uint32).reshape(-1, 3)
    return v, t


def sweep(verts, tris, theta_deg, phi_deg, freqs_hz, nx, ny, grid_size, max_bounces,
          reflection_const=1.0, precision=64, accel="tree", threads=0, records=False,
          model_scale=1.0, amb_edge=1e-6, amb_t=1e-6, amb_det=1e-3) -> SweepOut:
    """Reference-semantics sweep on the CPU oracle."""
    v, t = _mesh_args(verts, tris)
    th = np.ascontiguousarray(theta_deg, dtype=np.float64).ravel()
    ph = np.ascontiguousarray(phi_deg, dtype=np.float64).ravel()
    fr = np.ascontiguousarray(np.atleast_1d(freqs_hz), dtype=np.float64)
    na, nf = th.size, fr.size
    re = np.zeros(na * nf)
    im = np.zeros(na * nf)
    counts = np.zeros(na, dtype=COUNTS)
    rays = np.zeros((na, ny, nx), dtype=ORACLE_RAY) if records else None
    rc = lib().oracle_sweep(
        _ptr(v), v.shape[0], _ptr(t), t.shape[0], float(model_scale),
        _ptr(th), _ptr(ph), na, _ptr(fr), nf,
        int(nx), int(ny), float(grid_size), int(max_bounces), float(reflection_const),
        int(precision), 1 if accel == "tree" else 0, int(threads), _ptr(re), _ptr(im),
        _ptr(counts), _ptr(rays), float(amb_edge), float(amb_t), float(amb_det),
    )
    if rc != 0:
        raise RuntimeError(f"oracle_sweep failed with code {rc}")
    return SweepOut((re + 1j * im).reshape(na, nf), counts, rays)


def trace_rays(verts, tris, theta_deg, phi_deg, rays, nx, ny, grid_size, max_bounces, precision=64,
               accel="brute", threads=0, records=True, model_scale=1.0, amb_edge=1e-6, amb_t=1e-6, amb_det=1e-3):
    """Traces only the listed rays: rays[k] = (angle index, i, j) on the nx x ny
    launcher of that angle.  Returns (records [n] or None, COUNTS totals)."""
    v, t = _mesh_args(verts, tris)
    th = np.ascontiguousarray(theta_deg, dtype=np.float64).ravel()
    ph = np.ascontiguousarray(phi_deg, dtype=np.float64).ravel()
    rl = np.ascontiguousarray(rays, dtype=np.int32).reshape(-1, 3)
    out = np.zeros(rl.shape[0], dtype=ORACLE_RAY) if records else None
    counts = np.zeros(1, dtype=COUNTS)
    rc = lib().oracle_trace_rays(
        _ptr(v), v.shape[0], _ptr(t), t.shape[0], float(model_scale),
        _ptr(th), _ptr(ph), th.size, _ptr(rl), rl.shape[0],
        int(nx), int(ny), float(grid_size), int(max_bounces), int(precision),
        1 if accel == "tree" else 0, int(threads), _ptr(out), _ptr(counts),
        float(amb_edge), float(amb_t), float(amb_det),
    )
    if rc != 0:
        raise RuntimeError(f"oracle_trace_rays failed with code {rc}")
    return out, counts[0]


def sweep_pol(verts, tris, theta_deg, phi_deg, freqs_hz, nx, ny, grid_size, max_bounces,
              reflection_const=1.0, accel="tree", threads=0, model_scale=1.0) -> np.ndarray:
    """Polarised FP64 sweep (E-vector tracking, physical exit path; no reference
    counterpart): complex128 [n_angles, n_freqs, 2] with (HH, VV) last."""
    v, t = _mesh_args(verts, tris)
    th = np.ascontiguousarray(theta_deg, dtype=np.float64).ravel()
    ph = np.ascontiguousarray(phi_deg, dtype=np.float64).ravel()
    fr = np.ascontiguousarray(np.atleast_1d(freqs_hz), dtype=np.float64)
    na, nf = th.size, fr.size
    re = np.zeros(na * nf * 2)
    im = np.zeros(na * nf * 2)
    rc = lib().oracle_sweep_pol(
        _ptr(v), v.shape[0], _ptr(t), t.shape[0], float(model_scale),
        _ptr(th), _ptr(ph), na, _ptr(fr), nf,
        int(nx), int(ny), float(grid_size), int(max_bounces), float(reflection_const),
        1 if accel == "tree" else 0, int(threads), _ptr(re), _ptr(im),
    )
    if rc != 0:
        raise RuntimeError(f"oracle_sweep_pol failed with code {rc}")
    return (re + 1j * im).reshape(na, nf, 2)


def ref_sweep(verts, tris, theta_deg, phi_deg, freqs_hz, nx, ny, grid_size, max_bounces,
              reflection_const=1.0, kind=64, threads=0, records=False, model_scale=1.0) -> SweepOut:
    """The reference's own per-ray routine (oracle/_ref) on the host cores."""
    v, t = _mesh_args(verts, tris)
    th = np.ascontiguousarray(theta_deg, dtype=np.float64).ravel()
    ph = np.ascontiguousarray(phi_deg, dtype=np.float64).ravel()
    fr = np.ascontiguousarray(np.atleast_1d(freqs_hz), dtype=np.float64)
    na, nf = th.size, fr.size
    re = np.zeros(na * nf)
    im = np.zeros(na * nf)
    bounces = np.zeros(na, dtype=np.uint64)
    rays = np.zeros((na, ny, nx), dtype=REF_RAY) if records else None
    rc = ref_lib(kind).ref_sweep(
        _ptr(v), v.shape[0], _ptr(t), t.shape[0], float(model_scale),
        _ptr(th), _ptr(ph), na, _ptr(fr), nf,
        int(nx), int(ny), float(grid_size), int(max_bounces), float(reflection_const), int(threads),
        _ptr(re), _ptr(im), _ptr(bounces), _ptr(rays),
    )
    if rc != 0:
        raise RuntimeError(f"ref_sweep failed with code {rc}")
    counts = np.zeros(na, dtype=COUNTS)
    counts["bounces"] = bounces
    counts["rays"] = nx * ny
    return SweepOut((re + 1j * im).reshape(na, nf), counts, rays)


class RefScene:
    """The reference's SAH tree of one mesh, built once (oracle/_ref), for timing
    bounded row samples of a sweep with the reference's own per-ray routine."""

    def __init__(self, verts, tris, kind="32fast", model_scale=1.0):
        v, t = _mesh_args(verts, tris)
        self._L = ref_lib(kind)
        t0 = time.perf_counter()
        self._h = self._L.ref_scene_create(_ptr(v), v.shape[0], _ptr(t), t.shape[0], float(model_scale))
        self.build_s = time.perf_counter() - t0
        if not self._h:
            raise RuntimeError("reference tree build failed")

    def trace_rows(self, theta_deg, phi_deg, rows, freqs_hz, grid_size, max_bounces, reflection_const=1.0,
                   threads=0):
        """rows[k] = (angle index, n, j): row j of the n x n launcher of that angle,
        at frequency freqs_hz[k].  Returns (per-row complex PO sums, rays, bounces,
        seconds of tracing)."""
        th = np.ascontiguousarray(theta_deg, dtype=np.float64).ravel()
        ph = np.ascontiguousarray(phi_deg, dtype=np.float64).ravel()
        rl = np.ascontiguousarray(rows, dtype=np.int32).reshape(-1, 3)
        fr = np.ascontiguousarray(freqs_hz, dtype=np.float64).ravel()
        if fr.size != rl.shape[0]:
            raise ValueError("one frequency per row")
        re, im = np.zeros(rl.shape[0]), np.zeros(rl.shape[0])
        rays, bounces, secs = C.c_uint64(), C.c_uint64(), C.c_double()
        rc = self._L.ref_trace_rows(self._h, _ptr(th), _ptr(ph), th.size, _ptr(rl), rl.shape[0], _ptr(fr),
                                    float(grid_size), int(max_bounces), float(reflection_const), int(threads),
                                    _ptr(re), _ptr(im), C.byref(rays), C.byref(bounces), C.byref(secs))
        if rc != 0:
            raise RuntimeError(f"ref_trace_rows failed with code {rc}")
        return re + 1j * im, rays.value, bounces.value, secs.value

    def close(self):
        if self._h:
            self._L.ref_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


REF_LOAD_SO = os.path.join(HERE, "_ref", "libsbrrefload.so")


def ref_tree_root():
    """Root of the reference tree oracle/_ref was built from (None when it is not
    present on this machine)."""
    p = os.path.join(HERE, "_ref", "ref_root.txt")
    if not os.path.exists(p):
        return None
    root = open(p).read().strip()
    return root if root and os.path.isdir(root) else None


def ref_load_triangles(path: str, model_scale: float = 1.0) -> np.ndarray:
    """The reference's own loader (src/modelLoader.cpp) on `path`, de-indexed with the
    model scale as runRcsApp does in its FP32 build: float32 [ntris, 3, 3]."""
    L = C.CDLL(REF_LOAD_SO)
    L.ref_load_triangles.restype = C.c_int
    L.ref_load_triangles.argtypes = [C.c_char_p, _D, _P, _P, C.c_char_p, C.c_size_t]
    L.ref_free.argtypes = [_P]
    out, n = C.c_void_p(), C.c_size_t()
    err = C.create_string_buffer(1024)
    rc = L.ref_load_triangles(path.encode(), float(model_scale), C.byref(out), C.byref(n), err, 1024)
    if rc != 0:
        raise RuntimeError(f"reference loader failed ({rc}): {err.value.decode(errors='replace')}")
    arr = np.ctypeslib.as_array(C.cast(out, C.POINTER(C.c_float)), shape=(n.value * 9,)).copy()
    L.ref_free(out)
    return arr.reshape(-1, 3, 3)


def build_tree(verts, tris, model_scale=1.0, source="oracle"):
    """Reference SAH tree: (bounds [n,6], links [n,4], per-slot data)."""
    v, t = _mesh_args(verts, tris)
    n = t.shape[0]
    bounds = np.zeros((2 * n, 6))
    links = np.zeros((2 * n, 4), dtype=np.int32)
    if source == "oracle":
        order = np.zeros(n, dtype=np.int32)
        cnt = lib().oracle_build_tree(_ptr(v), v.shape[0], _ptr(t), n, float(model_scale),
                                      _ptr(bounds), _ptr(links), _ptr(order))
        extra = order
    else:
        tv = np.zeros((n, 9))
        cnt = ref_lib(64).ref_build_tree(_ptr(v), v.shape[0], _ptr(t), n, float(model_scale),
                                         _ptr(bounds), _ptr(links), _ptr(tv))
        extra = tv
    if cnt < 0:
        raise RuntimeError("tree build failed")
    return bounds[:cnt], links[:cnt], extra


def frame(theta_deg, phi_deg, grid_size):
    out = np.zeros(12)
    lib().oracle_frame(float(theta_deg), float(phi_deg), float(grid_size), _ptr(out))
    return {"dir": out[0:3], "u": out[3:6], "v": out[6:9], "llc": out[9:12]}


def aperture_rect(verts, theta_deg, phi_deg, nx, ny, grid_size):
    """Pixel rectangle (i0, i1, j0, j1), inclusive, of the projection of the mesh's
    bounding box on the launcher of one angle: the rays that can hit anything."""
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 3)
    lo, hi = v.min(axis=0), v.max(axis=0)
    f = frame(theta_deg, phi_deg, grid_size)
    corners = np.array([[hi[0] if c & 1 else lo[0], hi[1] if c & 2 else lo[1], hi[2] if c & 4 else lo[2]]
                        for c in range(8)]) - f["llc"]
    s = corners @ f["u"] / (f["u"] @ f["u"])
    t = corners @ f["v"] / (f["v"] @ f["v"])
    i0 = int(np.clip(np.floor(s.min() * nx - 0.5), 0, nx - 1))
    i1 = int(np.clip(np.ceil(s.max() * nx - 0.5), 0, nx - 1))
    j0 = int(np.clip(np.floor(t.min() * ny - 0.5), 0, ny - 1))
    j1 = int(np.clip(np.ceil(t.max() * ny - 0.5), 0, ny - 1))
    return i0, i1, j0, j1


def sample_rays(verts, theta_deg, phi_deg, nx, ny, grid_size, per_angle, seed=0):
    """Seeded rays (angle index, i, j), `per_angle` of them drawn uniformly inside each
    angle's aperture rectangle (aperture_rect)."""
    rng = np.random.default_rng(seed)
    out = []
    for a, (th, ph) in enumerate(zip(np.ravel(theta_deg), np.ravel(phi_deg))):
        i0, i1, j0, j1 = aperture_rect(verts, th, ph, nx, ny, grid_size)
        i = rng.integers(i0, i1 + 1, per_angle)
        j = rng.integers(j0, j1 + 1, per_angle)
        out.append(np.stack([np.full(per_angle, a), i, j], axis=1))
    return np.concatenate(out).astype(np.int32) if out else np.zeros((0, 3), np.int32)

