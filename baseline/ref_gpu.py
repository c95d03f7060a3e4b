"""ctypes front of the reference's OWN GPU sweep (runSweep with its RT and PO kernels,
src/app/sweep.cu, src/cuda/rtKernels.cu, src/cuda/poKernels.cu), compiled for sm_100a
by baseline/Makefile into baseline/_ref/ (FP32 build and -DUSE_DOUBLE build).

This is the reference arm beside the engine's numbers on the same GPU: one
launchRaysMultiBounce + integratePoMultiBounce pair per (angle, frequency), exactly
as the reference runs it.  It is not part of the engine and the engine never calls it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict[int, ctypes.CDLL] = {}

_d = ctypes.POINTER(ctypes.c_double)
_i32 = ctypes.POINTER(ctypes.c_int32)


def lib_path(bits: int = 32) -> str:
    return os.path.join(HERE, "_ref", f"libsbrrefgpu{bits}.so")


def available(bits: int = 32) -> bool:
    return os.path.exists(lib_path(bits))


def lib(bits: int = 32) -> ctypes.CDLL:
    if bits not in _LIBS:
        path = lib_path(bits)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C baseline with the reference tree present)")
        L = ctypes.CDLL(path)
        L.sbrref_gpu_real_bits.restype = ctypes.c_int
        L.sbrref_gpu_sweep.restype = ctypes.c_int
        L.sbrref_gpu_sweep.argtypes = [
            ctypes.POINTER(ctypes.c_float), ctypes.c_int64, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int64,
            ctypes.c_double, ctypes.c_int, _d, _i32, _i32, ctypes.c_double, ctypes.c_int, ctypes.c_double,
            ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
            _d, _d, _d, _d, _d, _d]
        if L.sbrref_gpu_real_bits() != bits:
            raise RuntimeError(f"{path} is not the {bits}-bit build")
        _LIBS[bits] = L
    return _LIBS[bits]


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def sweep(verts, tris, freqs, grids, G, max_bounces, R=1.0, theta=(90.0, 90.0, 1), phi=(0.0, 0.0, 1),
          bits=32, model_scale=1.0):
    """Run the reference's runSweep once per frequency on the current CUDA device.

    `theta` / `phi` are (start, end, samples) as in config.txt; `grids[i]` is the ray
    grid (nx = ny) of frequency i.  Returns a dict with the reference's own angles
    (theta outer, phi inner), sigma [n_freqs, n_angles] in m^2, the wall time of each
    runSweep call, the reference's own summed RT + PO kernel time per call (ms) and
    the BVH build time.
    """
    v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tris, dtype=np.uint32).reshape(-1, 3)
    f = np.ascontiguousarray(freqs, dtype=np.float64).ravel()
    n = np.ascontiguousarray(grids, dtype=np.int32).ravel()
    if n.size != f.size:
        raise ValueError("one grid per frequency")
    th0, th1, nth = float(theta[0]), float(theta[1]), int(theta[2])
    ph0, ph1, nph = float(phi[0]), float(phi[1]), int(phi[2])
    nang = nth * nph
    th_out = np.zeros(nang)
    ph_out = np.zeros(nang)
    sigma = np.zeros((f.size, nang))
    wall = np.zeros(f.size)
    kms = np.zeros(f.size)
    build = np.zeros(1)
    rc = lib(bits).sbrref_gpu_sweep(
        _ptr(v, ctypes.c_float), v.shape[0], _ptr(t, ctypes.c_uint32), t.shape[0], float(model_scale), f.size,
        _ptr(f, ctypes.c_double), _ptr(n, ctypes.c_int32), _ptr(n, ctypes.c_int32), float(G), int(max_bounces),
        float(R), th0, th1, nth, ph0, ph1, nph, _ptr(th_out, ctypes.c_double), _ptr(ph_out, ctypes.c_double),
        _ptr(sigma, ctypes.c_double), _ptr(wall, ctypes.c_double), _ptr(kms, ctypes.c_double),
        _ptr(build, ctypes.c_double))
    if rc != 0:
        raise RuntimeError(f"sbrref_gpu_sweep returned {rc}")
    return {"theta": th_out, "phi": ph_out, "sigma": sigma, "wall_s": wall, "kernel_ms": kms,
            "build_s": float(build[0])}
