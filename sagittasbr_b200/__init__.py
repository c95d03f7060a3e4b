"""sagittasbr_b200 -- B200-native SBR monostatic RCS engine (host side in Python).

The compute path is libsbr.so (sm_100a CUDA + C ABI, include/sbr.h).  This module
is a thin host mirror of the reference's interface for the hot path:

  reference                                   here
  ---------                                   ----
  loadConfig (src/app/config.cpp:39)          load_config()
  buildBvh + device upload                    Scene(...)
    (src/app/rtRcsEntry.cu:115-196)
  runSweep (src/app/sweep.cu:35)              run_sweep()  -> CSV rows + results
  launchRaysMultiBounce + integratePo...      run() / Plan (batched or per-angle)

It never computes anything itself: if libsbr.so is missing, every entry point
raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import (FIRST_HIT_AUTO, FIRST_HIT_RASTER, FIRST_HIT_TRAVERSE, MODE_BATCHED, MODE_PER_ANGLE, POL_HHVV, POL_SCALAR,
                   PREC_FP32, PREC_FP64, PREC_MIXED, SbrError, check, lib)

__all__ = [
    "Scene", "JobSpec", "SweepResult", "Plan", "run", "adjoint", "trace_records", "load_config", "config_angles",
    "load_obj", "load_gltf", "load_model", "write_csv", "run_sweep", "freq_scan", "SbrError", "MODE_BATCHED", "MODE_PER_ANGLE", "PREC_MIXED",
    "FIRST_HIT_AUTO", "FIRST_HIT_RASTER", "FIRST_HIT_TRAVERSE",
    "PREC_FP32", "PREC_FP64", "POL_SCALAR", "POL_HHVV", "RAY_RECORD",
]

RAY_RECORD = np.dtype(_lib.RAY_RECORD_FIELDS, align=True)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Scene:
    """Triangle mesh resident on one GPU with its BVH (sbr_scene_create)."""

    def __init__(self, verts, tris, model_scale: float = 1.0, device: int = -1, leaf_size: int = 0,
                 bin_count: int = 0, n_threads: int = 0, want_fp64: bool = False, gpu_build: bool = False,
                 node_width: int = 0):
        v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(tris, dtype=np.uint32).reshape(-1, 3)
        o = _lib.BuildOpts()
        o.model_scale = float(model_scale)
        o.device = int(device)
        o.leaf_size = int(leaf_size)
        o.bin_count = int(bin_count)
        o.n_threads = int(n_threads)
        o.want_fp64 = 1 if want_fp64 else 0
        o.gpu_build = 1 if gpu_build else 0
        o.node_width = int(node_width)
        h = C.c_void_p()
        check(lib().sbr_scene_create(_p(v), v.shape[0], _p(t), t.shape[0], C.byref(o), C.byref(h)),
              "sbr_scene_create")
        self._h = h
        self.n_triangles = t.shape[0]
        self.n_vertices = v.shape[0]

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("scene is closed")
        return self._h

    def info(self) -> dict:
        i = _lib.SceneInfo()
        check(lib().sbr_scene_info_get(self.handle, C.byref(i)), "sbr_scene_info_get")
        return {
            "n_triangles": i.n_triangles, "n_nodes_bin": i.n_nodes_bin, "n_nodes_gpu": i.n_nodes_gpu,
            "device_bytes": i.device_bytes, "aabb_lo": list(i.aabb_lo), "aabb_hi": list(i.aabb_hi),
            "build_ms": i.build_ms, "device": i.device, "bvh_depth": i.bvh_depth, "sah_ms": i.sah_ms,
        }

    def update_vertices(self, verts):
        """New vertex coordinates (same count and triangles); the BVH is refitted on
        the GPU (sbr_scene_update_vertices).  Create plans after the update."""
        v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
        check(lib().sbr_scene_update_vertices(self.handle, _p(v), v.shape[0]), "sbr_scene_update_vertices")

    def cancel(self):
        check(lib().sbr_scene_cancel(self.handle), "sbr_scene_cancel")

    def reset_cancel(self):
        check(lib().sbr_scene_reset_cancel(self.handle), "sbr_scene_reset_cancel")

    def close(self):
        if self._h is not None:
            check(lib().sbr_scene_destroy(self._h), "sbr_scene_destroy")
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class JobSpec:
    """Angles traced on one ray grid, with the frequencies that share it."""
    theta_deg: Sequence[float]
    phi_deg: Sequence[float]
    freqs_hz: Sequence[float]
    nx: int
    ny: int
    grid_size: float
    max_bounces: int
    reflection_const: float = 1.0
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> _lib.Job:
        th = np.ascontiguousarray(self.theta_deg, dtype=np.float64).ravel()
        ph = np.ascontiguousarray(self.phi_deg, dtype=np.float64).ravel()
        fr = np.ascontiguousarray(np.atleast_1d(self.freqs_hz), dtype=np.float64).ravel()
        if th.size != ph.size:
            raise ValueError("theta and phi lists differ in length")
        self._keep = [th, ph, fr]
        j = _lib.Job()
        j.theta_deg, j.phi_deg, j.n_angles = th.ctypes.data, ph.ctypes.data, th.size
        j.freq_hz, j.n_freqs = fr.ctypes.data, fr.size
        j.nx, j.ny, j.grid_size = int(self.nx), int(self.ny), float(self.grid_size)
        j.max_bounces, j.reflection_const = int(self.max_bounces), float(self.reflection_const)
        return j

    @property
    def n_angles(self):
        return len(np.atleast_1d(self.theta_deg))

    @property
    def n_freqs(self):
        return len(np.atleast_1d(self.freqs_hz))


@dataclass
class SweepResult:
    field: np.ndarray      # complex128 [n_samples] (job, angle, freq order); [n_samples, 2] (HH, VV) polarised
    sigma_m2: np.ndarray
    rcs_dbsm: np.ndarray
    stats: np.ndarray      # uint64 [n_job_angles, 4]: rays, hit rays, bounces, queries
    device_ms: float

    @property
    def bounces(self) -> int:
        return int(self.stats[:, 2].sum())

    @property
    def queries(self) -> int:
        return int(self.stats[:, 3].sum())


def _opts(mode, precision, polarization=POL_SCALAR, stream=None, use_graph=False, ctas_per_sm=0,
          first_hit=FIRST_HIT_AUTO, blocks_per_item=0, autotune=False, node_width=0, tile_cap=0):
    o = _lib.RunOpts()
    o.mode, o.precision, o.polarization = int(mode), int(precision), int(polarization)
    o.use_graph = 1 if use_graph else 0
    o.stream = stream
    o.ctas_per_sm = int(ctas_per_sm)
    o.first_hit = int(first_hit)
    o.blocks_per_item = int(blocks_per_item)
    o.autotune = 1 if autotune else 0
    o.node_width = int(node_width)
    o.tile_cap = int(tile_cap)
    return o


def _jobs_c(jobs):
    arr = (_lib.Job * len(jobs))()
    for i, j in enumerate(jobs):
        arr[i] = j.to_c()
    return arr


class Plan:
    """Prepared sweep (sbr_plan): frames, work items and result buffers on the GPU."""

    def __init__(self, scene: Scene | Sequence[Scene], jobs: Sequence[JobSpec], mode=MODE_BATCHED,
                 precision=PREC_MIXED, stream=None, use_graph=False, ctas_per_sm=0, first_hit=None,
                 polarization=POL_SCALAR, job_scene: Sequence[int] | None = None, blocks_per_item=0,
                 autotune=False, node_width=0, tile_cap=0):
        """With a list of scenes, job j traces scene[job_scene[j]] (sbr_plan_create_multi).
        autotune=True times candidate (blocks_per_item, ctas_per_sm) settings on a sample of
        the angles first and keeps the fastest (batched mode); info reports the choice.
        tile_cap: FIRST_HIT_RASTER's longest per-tile triangle list (0: 48, at most 1024)."""
        self.scene = scene
        self.jobs = list(jobs)
        self._jc = _jobs_c(self.jobs)
        o = _opts(mode, precision, polarization, stream=stream, use_graph=use_graph, ctas_per_sm=ctas_per_sm,
                  first_hit=FIRST_HIT_AUTO if first_hit is None else first_hit,
                  blocks_per_item=blocks_per_item, autotune=autotune, node_width=node_width, tile_cap=tile_cap)
        h = C.c_void_p()
        if isinstance(scene, Scene):
            check(lib().sbr_plan_create(scene.handle, self._jc, len(self.jobs), C.byref(o), C.byref(h)),
                  "sbr_plan_create")
        else:
            scenes = list(scene)
            js = np.ascontiguousarray(np.zeros(len(self.jobs)) if job_scene is None else job_scene, dtype=np.int32)
            if js.size != len(self.jobs):
                raise ValueError("job_scene needs one scene index per job")
            hs = (C.c_void_p * len(scenes))(*[sc.handle.value for sc in scenes])
            self._keep = (scenes, js, hs)
            check(lib().sbr_plan_create_multi(hs, len(scenes), _p(js), self._jc, len(self.jobs), C.byref(o),
                                              C.byref(h)), "sbr_plan_create_multi")
        self._h = h
        i = _lib.PlanInfo()
        check(lib().sbr_plan_info_get(h, C.byref(i)), "sbr_plan_info_get")
        self.info = {f: getattr(i, f) for f, _ in _lib.PlanInfo._fields_}

    def execute(self):
        check(lib().sbr_plan_execute(self._h), "sbr_plan_execute")

    def results(self) -> SweepResult:
        n = self.info["n_samples"]
        na = self.info["n_job_angles"]
        npol = self.info["n_pol"]
        f = np.zeros(2 * n * npol)
        s = np.zeros(n * npol)
        d = np.zeros(n * npol)
        st = np.zeros(4 * na, dtype=np.uint64)
        r = _lib.Result()
        r.field, r.sigma_m2, r.rcs_dbsm, r.stats = f.ctypes.data, s.ctypes.data, d.ctypes.data, st.ctypes.data
        check(lib().sbr_plan_results(self._h, C.byref(r)), "sbr_plan_results")
        return _result(f, s, d, st.reshape(na, 4), r.device_ms, npol)

    def device_results(self):
        pf, ps = C.c_void_p(), C.c_void_p()
        check(lib().sbr_plan_device_results(self._h, C.byref(pf), C.byref(ps)), "sbr_plan_device_results")
        return pf.value, ps.value

    def close(self):
        if self._h is not None:
            check(lib().sbr_plan_destroy(self._h), "sbr_plan_destroy")
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _result(f, s, d, st, ms, npol):
    field = f[0::2] + 1j * f[1::2]
    if npol > 1:
        field, s, d = field.reshape(-1, npol), s.reshape(-1, npol), d.reshape(-1, npol)
    return SweepResult(field, s, d, st, ms)


def run(scene: Scene, jobs: Sequence[JobSpec] | JobSpec, mode=MODE_BATCHED, precision=PREC_MIXED,
        stream=None, first_hit=None, polarization=POL_SCALAR, blocks_per_item=0, tile_cap=0) -> SweepResult:
    """One call through sbr_run: host arrays in, host arrays out.  With
    polarization=POL_HHVV the fields, sigma and dBsm carry a trailing (HH, VV) axis."""
    if isinstance(jobs, JobSpec):
        jobs = [jobs]
    jc = _jobs_c(jobs)
    npol = 2 if polarization == POL_HHVV else 1
    n = sum(j.n_angles * j.n_freqs for j in jobs)
    na = sum(j.n_angles for j in jobs)
    f = np.zeros(2 * n * npol)
    s = np.zeros(n * npol)
    d = np.zeros(n * npol)
    st = np.zeros(4 * na, dtype=np.uint64)
    r = _lib.Result()
    r.field, r.sigma_m2, r.rcs_dbsm, r.stats = f.ctypes.data, s.ctypes.data, d.ctypes.data, st.ctypes.data
    o = _opts(mode, precision, polarization, stream=stream,
              first_hit=FIRST_HIT_AUTO if first_hit is None else first_hit, blocks_per_item=blocks_per_item,
              tile_cap=tile_cap)
    check(lib().sbr_run(scene.handle, jc, len(jobs), C.byref(r), C.byref(o)), "sbr_run")
    return _result(f, s, d, st.reshape(na, 4), r.device_ms, npol)


def adjoint(scene: Scene, jobs: Sequence[JobSpec] | JobSpec, cot, precision=PREC_MIXED, stream=None):
    """sbr_adjoint: gradient of a loss of the sweep's fields along the frozen hit paths.

    cot: complex [n_samples] cotangent g of each sample's field S (dLoss =
    sum Re(conj(g) dS)).  Returns (grad_xyz [nverts, 3] with respect to the caller's
    vertex coordinates, grad_freq [n_samples] with respect to each sample's
    frequency in Hz)."""
    if isinstance(jobs, JobSpec):
        jobs = [jobs]
    jc = _jobs_c(jobs)
    n = sum(j.n_angles * j.n_freqs for j in jobs)
    g = np.ascontiguousarray(np.asarray(cot, dtype=np.complex128).ravel())
    if g.size != n:
        raise ValueError(f"cotangent has {g.size} entries, the jobs have {n} samples")
    c2 = np.ascontiguousarray(np.stack([g.real, g.imag], axis=1).ravel())
    gx = np.zeros(3 * scene.n_vertices)
    gf = np.zeros(n)
    o = _opts(MODE_BATCHED, precision, stream=stream)
    check(lib().sbr_adjoint(scene.handle, jc, len(jobs), C.byref(o), _p(c2), _p(gx), _p(gf)), "sbr_adjoint")
    return gx.reshape(-1, 3), gf


def trace_records(scene: Scene, job: JobSpec, precision=PREC_MIXED, first_hit=None, tile_cap=0) -> np.ndarray:
    """Per-ray hit records [n_angles, ny, nx] (sbr_trace_records)."""
    jc = job.to_c()
    out = np.zeros((job.n_angles, job.ny, job.nx), dtype=RAY_RECORD)
    o = _opts(MODE_BATCHED, precision, first_hit=FIRST_HIT_AUTO if first_hit is None else first_hit,
              tile_cap=tile_cap)
    check(lib().sbr_trace_records(scene.handle, C.byref(jc), C.byref(o), _p(out)), "sbr_trace_records")
    return out


def error_bound(scene: Scene, jobs: Sequence[JobSpec] | JobSpec, result: SweepResult, stream=None):
    """Stated error of a mixed-precision result against FP64 (sbr_error_bound):
    (bound on |field - field_FP64| [n_samples], bound on |dBsm - dBsm_FP64|
    [n_samples])."""
    if isinstance(jobs, JobSpec):
        jobs = [jobs]
    jc = _jobs_c(jobs)
    f = np.ascontiguousarray(np.stack([result.field.real, result.field.imag], axis=1).ravel())
    n = f.size // 2
    ef, ed = np.zeros(n), np.zeros(n)
    o = _opts(MODE_BATCHED, PREC_MIXED, stream=stream)
    check(lib().sbr_error_bound(scene.handle, jc, len(jobs), C.byref(o), _p(f), _p(ef), _p(ed)), "sbr_error_bound")
    return ef, ed


def trace_ray_list(scene: Scene, job: JobSpec, rays, precision=PREC_MIXED) -> np.ndarray:
    """Hit records [n] of the listed rays only, rays[k] = (angle index, i, j)
    (sbr_trace_ray_list)."""
    jc = job.to_c()
    rl = np.ascontiguousarray(rays, dtype=np.int32).reshape(-1, 3)
    out = np.zeros(rl.shape[0], dtype=RAY_RECORD)
    o = _opts(MODE_BATCHED, precision)
    check(lib().sbr_trace_ray_list(scene.handle, C.byref(jc), C.byref(o), _p(rl), rl.shape[0], _p(out)),
          "sbr_trace_ray_list")
    return out


# ------------------------------------------------------------ entry surface
def load_config(path: str = "config.txt", argv: Sequence[str] = ()) -> dict:
    """loadConfig(path, argc, argv): argv excludes the program name."""
    args = [b"RT-RCS"] + [a.encode() for a in argv]
    arr = (C.c_char_p * len(args))(*args)
    c = _lib.Config()
    check(lib().sbr_config_load(path.encode(), len(args), arr, C.byref(c)), "sbr_config_load")
    out = {f: getattr(c, f) for f, _ in _lib.Config._fields_}
    out["model_path"] = c.model_path.decode()
    out["_c"] = c
    return out


def _cfg_struct(cfg: dict) -> _lib.Config:
    c = _lib.Config()
    for f, _ in _lib.Config._fields_:
        if f == "model_path":
            c.model_path = cfg.get("model_path", "").encode()
        elif f in cfg:
            setattr(c, f, cfg[f])
    return c


def config_angles(cfg: dict):
    n = max(0, cfg["theta_samples"]) * max(0, cfg["phi_samples"])
    th = np.zeros(n)
    ph = np.zeros(n)
    c = _cfg_struct(cfg)
    check(lib().sbr_config_angles(C.byref(c), _p(th), _p(ph)), "sbr_config_angles")
    return th, ph


def load_obj(path: str):
    """OBJ mesh -> (verts float32 [V, 3], tris uint32 [T, 3]) (sbr_load_obj)."""
    return _load("sbr_load_obj", path)


def load_gltf(path: str):
    """glTF 2.0 / GLB mesh -> (verts, tris) (sbr_load_gltf)."""
    return _load("sbr_load_gltf", path)


def load_model(path: str):
    """loadModel: .obj, .gltf or .glb by extension (sbr_load_model)."""
    return _load("sbr_load_model", path)


def _load(fn: str, path: str):
    pv, pt = C.c_void_p(), C.c_void_p()
    nv, nt = C.c_size_t(), C.c_size_t()
    check(getattr(lib(), fn)(path.encode(), C.byref(pv), C.byref(nv), C.byref(pt), C.byref(nt)), fn)
    try:
        v = np.ctypeslib.as_array(C.cast(pv, C.POINTER(C.c_float)), shape=(nv.value * 3,)).copy()
        t = np.ctypeslib.as_array(C.cast(pt, C.POINTER(C.c_uint32)), shape=(nt.value * 3,)).copy()
    finally:
        lib().sbr_free(pv)
        lib().sbr_free(pt)
    return v.reshape(-1, 3), t.reshape(-1, 3)


def write_csv(path: str, cfg: dict, theta, phi, sigma, dbsm, err_db=None):
    """rcs_results.csv in the reference layout; with err_db a fifth column rcs_err_db."""
    c = _cfg_struct(cfg)
    th, ph = np.ascontiguousarray(theta, np.float64), np.ascontiguousarray(phi, np.float64)
    s, d = np.ascontiguousarray(sigma, np.float64), np.ascontiguousarray(dbsm, np.float64)
    if err_db is None:
        check(lib().sbr_write_csv(path.encode(), C.byref(c), _p(th), _p(ph), _p(s), _p(d), th.size),
              "sbr_write_csv")
    else:
        e = np.ascontiguousarray(err_db, np.float64)
        check(lib().sbr_write_csv_err(path.encode(), C.byref(c), _p(th), _p(ph), _p(s), _p(d), _p(e), th.size),
              "sbr_write_csv_err")


def run_sweep(cfg: dict, scene: Scene, out_csv: str | None = "rcs_results.csv", mode=None, precision=None):
    """runSweep (src/app/sweep.cu:35): the config's theta x phi sweep at cfg['freq'],
    written to rcs_results.csv rows (theta-major).  Returns (theta, phi, SweepResult)."""
    th, ph = config_angles(cfg)
    job = JobSpec(th, ph, [cfg["freq"]], cfg["nx"], cfg["ny"], cfg["grid_size"], cfg["max_bounces"],
                  cfg["reflection_const"])
    prec = cfg.get("precision", PREC_MIXED) if precision is None else precision
    res = run(scene, job, mode=cfg.get("mode", MODE_BATCHED) if mode is None else mode, precision=prec)
    err = error_bound(scene, job, res)[1] if cfg.get("error_bound") and prec == PREC_MIXED else None
    if out_csv:
        write_csv(out_csv, cfg, th, ph, res.sigma_m2, res.rcs_dbsm, err)
    return th, ph, res


def freq_scan(cfg: dict, scene: Scene, f_start: float, f_end: float, n: int,
              out_csv: str | None = "results_freq_scans.csv", precision=None):
    """Frequency scan of the config's angle sweep (replaces util/run_freq_scan.sh:30-53
    with util/plotRCS.py --scans): frequencies round(logspace(f_start, f_end, n)) on
    the config's ray grid, traced as jobs of one plan (up to 128 frequencies share
    each angle's trace); returns (freqs, mean sigma, sample std of sigma) over the
    angles and appends them to `out_csv` (Frequency,Avg_RCS,Std_RCS)."""
    th, ph = config_angles(cfg)
    fr = np.round(np.logspace(np.log10(f_start), np.log10(f_end), n))
    jobs = [JobSpec(th, ph, fr[k:k + 128], cfg["nx"], cfg["ny"], cfg["grid_size"], cfg["max_bounces"],
                    cfg["reflection_const"]) for k in range(0, n, 128)]
    res = run(scene, jobs, precision=cfg.get("precision", PREC_MIXED) if precision is None else precision)
    blocks, off = [], 0
    for j in jobs:  # samples are job-major, then angle, then frequency
        m = th.size * j.n_freqs
        blocks.append(res.sigma_m2[off:off + m].reshape(th.size, j.n_freqs))
        off += m
    sig = np.concatenate(blocks, axis=1)
    mean = sig.mean(axis=0)
    std = sig.std(axis=0, ddof=1) if th.size > 1 else np.zeros_like(mean)
    if out_csv:
        import csv
        import os
        new = not os.path.exists(out_csv) or os.path.getsize(out_csv) == 0
        with open(out_csv, "a", newline="") as f:
            w = csv.writer(f)
            if new:
                w.writerow(["Frequency", "Avg_RCS", "Std_RCS"])
            for a, b, c in zip(fr, mean, std):
                w.writerow([float(a), float(b), float(c)])
    return fr, mean, std
