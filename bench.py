"""Benchmark of the SBR hot path on B200: angle-frequency samples/s and Mray-bounces/s.

Default workload (the sweep the >= 10x target is stated on, fits one GPU): seeded
procedural aircraft of 2,148,800 triangles (superellipsoid fuselage 20 m x 1.5 m,
swept trapezoidal wings of 18 m span and 3 -> 1 m chord, tail; Gaussian vertex jitter
1 mm), 64 frequencies log-spaced over 1-18 GHz, 721 azimuths at 0.5 deg (theta = 90),
max 5 bounces, 10 rays per wavelength over the bounding aperture (G = 20.36 m; all
frequencies share one trace on the 12,222^2 grid of 18 GHz); the primary rays' first
hits come from the tile-binned raster (the plan's automatic choice for this dense
sweep), every later bounce from the persistent trace, chunk by chunk of angles.
Other workloads (--workload): `trihedral` (3 x 100x100x2 triangles, 10 GHz, 578^2
rays, 3 bounces, theta, phi = 0..90 at 1 deg = 8,281 angles), `sphere` (icosphere
level 5, 1 GHz, 67^2 rays, 3 bounces, 360 azimuths), `aircraft-dev` (8 frequencies x
73 azimuths of the aircraft), `ellipsoid` (ellipsoid 2/1/0.5 m with a seeded 32-mode
spherical-harmonic displacement, 199,808 triangles, 5 GHz, G = 4 m, 668^2 rays,
4 bounces, 121 azimuths over -30..30 deg; --adjoint also times the gradient of the
mean RCS) and `uneven` (64 seeded meshes of 1k-500k triangles -- icospheres,
trihedrals, jittered ellipsoids, plate clusters -- each with its own frequency in
1-12 GHz, 90-1440 azimuths, 2-6 bounces and ray grid, drained by one graph-captured
launch of a multi-scene plan).  All meshes are synthetic and seeded; no dataset is
involved.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one full sweep of the workload.
`value`      whole-job samples/s of the batched engine with the plan resident in HBM
             (sbr_plan_execute on a torch stream, CUDA events, L2 flushed by a 256 MiB
             write before every step, inside the timed region).
`e2e`        the same metric through sbr_run with host arrays in and out (angle and
             frequency tables up, fields down), wall clock, median (and mean) of the
             calls after one untimed call.
`per_angle`  the engine in the reference's loop structure: one trace + PO launch per
             (angle, frequency), each frequency on its own grid n_f = ceil(10 G f / c),
             FP32 arithmetic -- the denominator of the >= 10x target -- on every 8th angle.
`reference_gpu` the reference's OWN GPU sweep (runSweep with its RT and PO kernels),
             compiled for sm_100a from its sources (baseline/Makefile), timed on the same
             GPU on a grid of angles; its USE_DOUBLE build is compared with the engine.
`fp64_check` batched mixed precision against a full-FP64 run of the same batched job
             on evenly spread angles: max |d dB| over every sample (unfiltered) and over
             the samples within 30 dB of each frequency's peak.
`roofline`   dominant kernel (k_trace): algorithmic FP32 work per closest-hit query
             on the reference SAH tree, 27 V_box + 57 V_tri FLOP, V_box / V_tri counted
             by the CPU oracle walking the reference tree on a seeded sample of the rays
             the engine launches; peak = FP32 SGEMM throughput measured in the same run
             (the peaks file holds HBM and bf16 figures only).
`cpu_baseline` the reference's own per-ray routine (src/cuda/rtKernels.cu) compiled
             for the host (oracle/_ref), OpenMP over all host cores, on a bounded
             uniform sample of the ray rows of the sweep (each (angle, frequency) on its
             own grid as the reference runs it); samples/s = samples / (rows of the
             sweep x measured seconds per row).
Under torchrun (N > 1) the one sweep is split: every rank traces its cost-balanced
shard of the angles (sharding.ShardedPlan) and the fields are gathered to rank 0
inside the timed region (strong scaling); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

C0 = 299792458.0
FLOP_PER_BOX = 27
FLOP_PER_TRI = 57


def workload(name: str):
    """Mesh, angles, frequencies and ray grids of a benchmark workload."""
    from sagittasbr_b200 import meshes as M
    if name == "trihedral":
        v, t = M.trihedral(1.0, 100)
        th, ph = np.meshgrid(np.arange(0.0, 91.0), np.arange(0.0, 91.0), indexing="ij")
        th, ph = th.ravel(), ph.ravel()
        freqs, mb = [1e10], 3
    elif name == "sphere":
        v, t = M.icosphere(5, 1.0)
        ph = np.arange(0.0, 360.0)
        th = np.full(ph.size, 90.0)
        freqs, mb = [1e9], 3
    elif name in ("aircraft", "aircraft-dev"):
        v, t = M.aircraft(seed=1)
        nf, step = (64, 0.5) if name == "aircraft" else (8, 5.0)
        ph = np.arange(0.0, 360.0 + 1e-9, step)
        th = np.full(ph.size, 90.0)
        freqs, mb = list(np.geomspace(1e9, 18e9, nf)), 5
    elif name == "ellipsoid":
        # differentiable-shape case: SH-displaced ellipsoid 2/1/0.5 m, 5 GHz, G = 4 m
        v, t = M.ellipsoid_sh()
        ph = np.arange(-30.0, 30.0 + 1e-9, 0.5)
        th = np.full(ph.size, 90.0)
        freqs, mb = [5e9], 4
    else:
        raise ValueError(name)
    G = 4.0 if name == "ellipsoid" else 2.0 * M.bounding_radius(v)
    grid = {f: M.rays_for(f, G) for f in freqs}
    n = grid[max(freqs)]
    label = f"{name}_{t.shape[0]}tri_{len(freqs)}f_{min(freqs)/1e9:g}-{max(freqs)/1e9:g}GHz_{n}x{n}_{mb}b_{th.size}ang"
    return dict(verts=v, tris=t, theta=th, phi=ph, freqs=freqs, grid=grid, nx=n, ny=n, G=G, max_bounces=mb,
                R=1.0, name=label, workload=name)


# (theta, phi) grids, as (start, end, samples), on which the reference's own GPU build
# is run: the timed sample (its own ray grid per frequency) and the FP64-build sample
# (the batched grid for every frequency) compared with the engine
REF_GPU_SAMPLES = {
    "trihedral": (((0.0, 90.0, 91), (0.0, 88.0, 12)), ((0.0, 90.0, 8), (0.0, 90.0, 8))),
    "sphere": (((90.0, 90.0, 1), (0.0, 352.0, 45)), ((90.0, 90.0, 1), (0.0, 350.0, 36))),
    "aircraft": (((90.0, 90.0, 1), (0.0, 360.0, 91)), ((90.0, 90.0, 1), (0.0, 315.0, 8))),
    "aircraft-dev": (((90.0, 90.0, 1), (0.0, 360.0, 73)), ((90.0, 90.0, 1), (0.0, 315.0, 8))),
    "ellipsoid": (((90.0, 90.0, 1), (-30.0, 30.0, 121)), ((90.0, 90.0, 1), (-30.0, 30.0, 25))),
}


def ref_gpu_leg(w, sbr, scene, value):
    """The reference's own GPU sweep (runSweep, FP32 build) timed on the same GPU, and
    its USE_DOUBLE build compared with the engine's batched mixed-precision result."""
    from baseline import ref_gpu
    if not ref_gpu.available(32):
        return {"unavailable": "baseline/_ref/libsbrrefgpu32.so not built (make -C baseline)"}
    (th, ph), (th64, ph64) = REF_GPU_SAMPLES[w["workload"]]
    freqs = w["freqs"]
    nf = len(freqs)
    r = ref_gpu.sweep(w["verts"], w["tris"], freqs, [w["grid"][f] for f in freqs], w["G"], w["max_bounces"],
                      w["R"], th, ph, bits=32)
    n = r["sigma"].size
    wall, kern = float(r["wall_s"].sum()), float(r["kernel_ms"].sum())
    out = {"value": n / wall, "unit": "samples/s", "samples": n, "angles": th[2] * ph[2], "freqs": nf,
           "theta": list(th), "phi": list(ph), "wall_s": wall,
           "kernel_only_value": n / (kern * 1e-3) if kern > 0 else None,
           "batched_speedup": value / (n / wall),
           "grids": "own grid per frequency, n_f = ceil(10 G f / c)",
           "what": "the reference's runSweep (launchRaysMultiBounce + integratePoMultiBounce per angle and "
                   "frequency, float atomics), FP32 build (--use_fast_math) compiled for sm_100a, one rank; "
                   "value = samples / wall time of its runSweep calls"}
    if ref_gpu.available(64):
        r64 = ref_gpu.sweep(w["verts"], w["tris"], freqs, [w["nx"]] * nf, w["G"], w["max_bounces"], w["R"],
                            th64, ph64, bits=64)
        job = sbr.JobSpec(r64["theta"], r64["phi"], freqs, w["nx"], w["ny"], w["G"], w["max_bounces"], w["R"])
        ours = sbr.run(scene, job, mode=sbr.MODE_BATCHED, precision=sbr.PREC_MIXED)
        ours64 = sbr.run(scene, job, mode=sbr.MODE_BATCHED, precision=sbr.PREC_FP64)
        ref_s = r64["sigma"].T  # [angle, freq], the engine's order
        db_ref = 10 * np.log10(np.maximum(ref_s, 1e-10))
        db = 10 * np.log10(np.maximum(ours.sigma_m2.reshape(ref_s.shape), 1e-10))
        db64 = 10 * np.log10(np.maximum(ours64.sigma_m2.reshape(ref_s.shape), 1e-10))
        lit = db_ref > db_ref.max(axis=0)[None, :] - 30.0
        d, d64 = np.abs(db - db_ref), np.abs(db64 - db_ref)
        # the engine's stated error of its mixed result against FP64 on the same samples
        _, ed = sbr.error_bound(scene, job, ours)
        ed = ed.reshape(ref_s.shape)
        over = d > 0.1
        out["fp64_build_vs_engine"] = {
            "samples": int(ref_s.size), "theta": list(th64), "phi": list(ph64), "grid": w["nx"],
            "mixed_max_abs_ddb": float(d.max()), "mixed_frac_within_0.1dB": float((d <= 0.1).mean()),
            "mixed_max_abs_ddb_within_30dB_of_peak": float(d[lit].max()),
            "fp64_max_abs_ddb": float(d64.max()),
            "mixed_samples_over_0.1dB": int(over.sum()),
            "mixed_over_0.1dB_within_stated_error_plus_fp64_gap": int((d[over] <= ed[over] + d64[over] + 1e-9).sum()),
            "mixed_over_0.1dB_detail": [{"ddb": float(d[q]), "stated_db": float(ed[q]), "fp64_gap_db": float(d64[q]),
                                         "dbsm_ref": float(db_ref[q]), "db_below_peak": float(
                                             db_ref.max(axis=0)[q[1]] - db_ref[q])}
                                        for q in zip(*np.nonzero(over))][:8],
            "fp64_max_rel_sigma_diff_within_30dB_of_peak": float(
                (np.abs(ours64.sigma_m2.reshape(ref_s.shape) - ref_s) / ref_s)[lit].max()),
            "ref_fp64_wall_s": float(r64["wall_s"].sum())}
    return out


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, val in zip(names, r[5:9]):
                    if val.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def fp32_peak_tflops(torch) -> float:
    """Dense FP32 (no TF32) SGEMM throughput at 8192^3: after a second of warm-up
    GEMMs, the best of 10 bursts of three back-to-back GEMMs."""
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda")
    b = torch.randn(n, n, device="cuda")
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < 1.0:
        a @ b
        torch.cuda.synchronize()
    best = 0.0
    for _ in range(10):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(3):
            a @ b
        e.record()
        e.synchronize()
        best = max(best, 3 * 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


def fma_peak_tflops(torch, sm_mhz: float) -> float:
    """The FP32 FMA issue rate of the device at a given SM clock: SMs x 128 FP32
    lanes x 2 FLOP per cycle."""
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    return sms * 128 * 2 * sm_mhz * 1e6 / 1e12


def config_of(w) -> dict:
    """The workload-defining keys of a bench line, identical in both arms."""
    return {"workload": w["name"], "angles": int(w["theta"].size), "freqs": len(w["freqs"]),
            "triangles": int(w["tris"].shape[0]), "rays_per_angle": int(w["nx"] * w["ny"]),
            "max_bounces": int(w["max_bounces"]), "grid_size_m": float(w["G"]),
            "freq_ghz": [float(min(w["freqs"])) / 1e9, float(max(w["freqs"])) / 1e9],
            "l2": "flushed before every step (256 MiB write inside the timed region)"}


def sweep_rows(w) -> int:
    """Ray rows of the sweep as the reference runs it: every (angle, frequency) on its
    own n_f x n_f grid."""
    return int(w["theta"].size) * int(sum(w["grid"][f] for f in w["freqs"]))


def draw_rows(w, rng, n):
    """n ray rows drawn uniformly from all rows of the sweep: (angle, n_f, row) and the
    row's frequency."""
    nf = np.array([w["grid"][f] for f in w["freqs"]], dtype=np.int64)
    fi = rng.choice(nf.size, n, p=nf / nf.sum())
    a = rng.integers(0, w["theta"].size, n)
    j = (rng.random(n) * nf[fi]).astype(np.int64)
    return np.stack([a, nf[fi], j], axis=1), np.asarray(w["freqs"], dtype=np.float64)[fi]


class CpuReference:
    """The reference's own per-ray routine compiled for the host (oracle/_ref, FP32,
    its release flags) on all host cores, timed on uniform samples of the sweep's ray
    rows; the reference tree is built once and not timed."""

    def __init__(self, w, threads: int = 0):
        from oracle import oracle as O
        if not O.ref_available("32fast"):
            raise RuntimeError("oracle/_ref/libsbrref32_fast.so is not built (make -C oracle with the reference)")
        self.w, self.threads = w, threads or (os.cpu_count() or 1)
        self.scene = O.RefScene(w["verts"], w["tris"], kind="32fast")
        self.rng = np.random.default_rng(7)

    def sample(self, budget_s: float) -> dict:
        """Rows traced until `budget_s` of tracing; samples/s estimated as the sweep's
        samples over (rows of the sweep x seconds per traced row)."""
        w = self.w
        rows_done = rays = bounces = 0
        secs = 0.0
        batch = 2 * self.threads
        while secs < budget_s:
            rows, fr = draw_rows(w, self.rng, batch)
            _, r, b, t = self.scene.trace_rows(w["theta"], w["phi"], rows, fr, w["G"], w["max_bounces"], w["R"],
                                               threads=self.threads)
            rows_done += rows.shape[0]
            rays += r
            bounces += b
            secs += t
        per_row = secs / rows_done
        sweep_s = sweep_rows(w) * per_row
        return {"value": w["theta"].size * len(w["freqs"]) / sweep_s, "rows": rows_done, "rays": rays,
                "seconds": secs, "rays_per_s": rays / secs, "mray_bounces_per_s": bounces / secs / 1e6,
                "sample": (f"{rows_done} ray rows drawn uniformly from the {sweep_rows(w)} rows of the sweep (each "
                           f"(angle, frequency) on its own n_f x n_f grid, as the reference runs it), {rays} rays; "
                           f"samples/s = {w['theta'].size * len(w['freqs'])} samples / (rows x measured s per row); "
                           f"reference rtKernels.cu host build (oracle/_ref, FP32, -O3), reference tree built once "
                           f"({self.scene.build_s:.1f} s, not timed)")}


def oracle_counts(w, n_angles: int = 8, per_angle: int = 512, threads: int = 0):
    """V_box and V_tri per closest-hit query on the reference SAH tree (leaf 4, 16
    bins), counted by the FP64 oracle on a seeded sample of the rays the engine
    launches: `per_angle` rays inside the clipped aperture of each of `n_angles`
    angles spread over the sweep, on the batched grid."""
    from oracle import oracle as O
    pick = np.unique(np.linspace(0, w["theta"].size - 1, n_angles).round().astype(int))
    th, ph = w["theta"][pick], w["phi"][pick]
    rays = O.sample_rays(w["verts"], th, ph, w["nx"], w["ny"], w["G"], per_angle, seed=11)
    t0 = time.perf_counter()
    _, c = O.trace_rays(w["verts"], w["tris"], th, ph, rays, w["nx"], w["ny"], w["G"], w["max_bounces"],
                        precision=64, accel="tree", threads=threads, records=False)
    q = float(c["queries"])
    return {"v_box": float(c["box_tests"]) / q, "v_tri": float(c["tri_tests"]) / q, "rays": int(rays.shape[0]),
            "angles": int(pick.size), "queries": int(q), "oracle_s": time.perf_counter() - t0}


# DRAM bytes per closest-hit query of k_trace, from one ncu capture per workload
# (dram__bytes_read.sum + dram__bytes_write.sum of one launch / the closest-hit
# queries of that launch), scaled by the queries of a full launch:
#   aircraft: 8 of the 721 azimuths, 64 frequencies, one launch: 709.2 MB read +
#             144.0 MB written for 4.253e8 queries;
#   trihedral: 64 of the 8,281 angles, one launch: 4.82 MB + 1.25 MB for 2.96e7 queries.
# measured DRAM bytes (read + write) per closest-hit query of the sweep's kernels
# (profiles/), by workload and first-hit mode: the raster adds the first-hit buffer
# (8 B per ray, written and read) and the tile lists to the trace's own traffic
DRAM_BYTES_PER_QUERY = {("aircraft", "walk"): 2.006, ("aircraft", "tile raster"): 15.39, ("trihedral", "walk"): 0.205}


def hbm_peak_gbs() -> tuple[float, str]:
    """Measured HBM copy bandwidth of this pool's B200s, else the earlier measurement."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        for k in ("hbm_gbs", "hbm_GBs", "hbm"):
            if k in d:
                return float(d[k]), "measured (peaks file)"
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback 6.65 TB/s (earlier measurement on this pool)"


def run_reference_arm(args):
    """The reference's own CPU implementation of the path (its per-ray routine,
    oracle/_ref) on the host cores: every step is a bounded sample of the workload's
    ray rows; rank 0 alone runs under torchrun."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    w = workload(args.workload)
    ref = CpuReference(w)
    budget = max(1.0, min(4.0, 90.0 / max(1, args.steps + args.warmup)))
    vals, ms, bps, last = [], [], [], None
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        last = ref.sample(budget)
        dt = (time.perf_counter() - t0) * 1e3
        if s >= args.warmup:
            vals.append(last["value"])
            ms.append(dt)
            bps.append(last["mray_bounces_per_s"])
    v = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": "angle-freq samples/s", "value": v, "unit": "samples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.mean(ms)), "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak",
        "vs_baseline": None, "dtype": "f32", "data": f"synthetic (seeded {args.workload} mesh)",
        "config": config_of(w),
        "step": "one bounded sample of the sweep's ray rows traced by the reference's per-ray routine "
                f"(about {budget:.1f} s of tracing); value = samples/s of the whole sweep estimated from it",
        "mray_bounces_per_s": float(np.mean(bps)),
        "cpu_baseline": {"value": v, "unit": "samples/s", "cores": ref.threads, "kind": "reference",
                         "sample": last["sample"]},
        "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_uneven(args, torch, sbr, dist, ws, rank, local):
    """The uneven batch: 64 seeded meshes of 1k-500k triangles, each with its own
    frequency, angle sweep, bounce limit and ray grid, all drained by one
    persistent launch of a multi-scene plan.  Under torchrun the instances are
    split across ranks by estimated cost (rays x bounces); the whole batch is the
    job (strong scaling)."""
    from sagittasbr_b200 import meshes as M
    from sagittasbr_b200.sharding import cost_partition
    batch = M.uneven_batch()
    cost = [b["n"] ** 2 * len(b["phi"]) * b["max_bounces"] for b in batch]
    start, count = cost_partition(cost, ws)[rank]
    mine = batch[start:start + count]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    t0 = time.perf_counter()
    scenes = [sbr.Scene(b["verts"], b["tris"], device=local) for b in mine]
    scene_s = time.perf_counter() - t0
    jobs = [sbr.JobSpec(b["theta"], b["phi"], [b["freq"]], b["n"], b["n"], b["G"], b["max_bounces"]) for b in mine]
    js = list(range(len(mine)))
    plan = sbr.Plan(scenes, jobs, precision=sbr.PREC_MIXED, stream=sp, use_graph=True, job_scene=js,
                    autotune=args.autotune)
    info = plan.info
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        flush.zero_()
        plan.execute()
    res = plan.results()
    barrier()
    clocks = Clocks(local) if rank == 0 else None
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for _ in range(args.steps):
        flush.zero_()
        plan.execute()
    t_end.record(stream)
    barrier()
    clk = clocks.stop() if clocks else None
    ms = torch.tensor([t_start.elapsed_time(t_end) / args.steps], device="cuda", dtype=torch.float64)
    # end to end through the public API: plan from host arrays, execute, results to host
    e2e = []
    for s in range(1 + max(3, min(args.steps, 5))):
        torch.cuda.synchronize()
        a = time.perf_counter()
        p2 = sbr.Plan(scenes, jobs, precision=sbr.PREC_MIXED, stream=sp, job_scene=js,
                      blocks_per_item=info["blocks_per_item"], ctas_per_sm=info["ctas_per_sm"])
        p2.execute()
        r2 = p2.results()
        p2.close()
        if s:
            e2e.append((time.perf_counter() - a) * 1e3)
    assert np.array_equal(r2.field, res.field)
    e2e_t = torch.tensor([float(np.median(e2e))], device="cuda", dtype=torch.float64)
    n_total = torch.tensor([float(info["n_samples"])], device="cuda", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n_total, op=dist.ReduceOp.SUM)
    step_ms, samples = float(ms[0]), float(n_total[0])
    # every instance against a full-FP64 run of eight of its angles: the four with
    # the strongest return in the batched sweep and four spread over the sweep.
    # Views where the return is far below the instance's peak (back faces of open
    # meshes, edge-on plates) are set by a few rays that touch edges, where the two
    # precisions may decide differently; the dB error is reported for samples
    # within 30 dB of the peak, and the field error relative to the peak field.
    per = []
    if args.fp64_check > 0:
        first = 0
        for b, sc, job in zip(mine, scenes, jobs):
            na = len(b["phi"])
            mag = np.abs(res.field[first:first + na])
            first += na
            pick = np.unique(np.concatenate([np.argsort(mag)[-4:], np.linspace(0, na - 1, 4).round().astype(int)]))
            cj = sbr.JobSpec(b["theta"][pick], b["phi"][pick], [b["freq"]], b["n"], b["n"], b["G"], b["max_bounces"])
            x = sbr.run(sc, cj, precision=sbr.PREC_MIXED)
            y = sbr.run(sc, cj, precision=sbr.PREC_FP64)
            ddb = np.abs(x.rcs_dbsm - y.rcs_dbsm)
            near = y.rcs_dbsm > y.rcs_dbsm.max() - 30.0
            per.append({"kind": b["kind"], "triangles": int(b["tris"].shape[0]), "max_abs_ddb": float(ddb.max()),
                        "max_abs_ddb_within_30dB_of_peak": float(ddb[near].max()),
                        "field_err_rel_to_peak": float(np.abs(x.field - y.field).max() / np.abs(y.field).max())})
    if dist is not None:
        dist.barrier()
    for sc in scenes:
        sc.close()
    if rank != 0:
        return 0
    tri = [int(b["tris"].shape[0]) for b in batch]
    line = {
        "metric": "angle-freq samples/s", "value": samples / (step_ms * 1e-3), "unit": "samples/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "fp32 traversal + fp32-pair phase + fp64 sums",
        "data": "synthetic (seeded uneven batch of 64 meshes)",
        "config": {"workload": f"uneven_64meshes_{min(tri)}-{max(tri)}tri_{int(sum(len(b['phi']) for b in batch))}samples",
                   "meshes": len(batch), "triangles_total": int(sum(tri)), "samples": int(samples),
                   "rays_launched_per_step": info["n_rays_clipped"], "mode": "batched persistent, multi-scene plan",
                   "cuda_graph": True, "precision": "mixed", "autotune": bool(args.autotune),
                   "blocks_per_item": info["blocks_per_item"], "ctas_per_sm": info["ctas_per_sm"],
                   "l2": "flushed before every step (256 MiB write inside the timed region)",
                   "parallelism": f"{ws} GPU(s), instances split by estimated cost", "scene_build_s": scene_s},
        "mray_bounces_per_s": res.bounces * ws / (step_ms * 1e-3) / 1e6,
        "e2e": {"value": samples / (float(e2e_t[0]) * 1e-3), "unit": "samples/s",
                "h2d_bytes_per_step": info["h2d_bytes"], "d2h_bytes_per_step": info["d2h_bytes"],
                "ms_per_step": float(e2e_t[0]), "note": "multi-scene plan built from host arrays each step"},
        "gpu_launches": int(info["launches_per_execute"]) * args.steps,
        "fp64_check": ({"instances": len(per),
                        "max_abs_ddb_within_30dB_of_peak": max(q["max_abs_ddb_within_30dB_of_peak"] for q in per),
                        "instances_within_0.1dB_near_peak": sum(q["max_abs_ddb_within_30dB_of_peak"] <= 0.1
                                                                for q in per),
                        "max_field_err_rel_to_peak": max(q["field_err_rel_to_peak"] for q in per),
                        "per_instance": per} if per else None),
        "roofline": None, "cpu_baseline": None, "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def fp64_check_leg(w, sbr, scene, n_angles: int) -> dict:
    """Batched mixed precision against a full-FP64 run of the same batched job on
    `n_angles` evenly spread angles, every frequency."""
    pick = np.unique(np.linspace(0, w["theta"].size - 1, n_angles).round().astype(int))
    cjob = sbr.JobSpec(w["theta"][pick], w["phi"][pick], w["freqs"], w["nx"], w["ny"], w["G"], w["max_bounces"],
                       w["R"])
    a = sbr.run(scene, cjob, mode=sbr.MODE_BATCHED, precision=sbr.PREC_MIXED)
    b = sbr.run(scene, cjob, mode=sbr.MODE_BATCHED, precision=sbr.PREC_FP64)
    t0 = time.perf_counter()
    ef, ed = sbr.error_bound(scene, cjob, a)
    bound_s = time.perf_counter() - t0
    ddb = np.abs(a.rcs_dbsm - b.rcs_dbsm)
    db64 = b.rcs_dbsm.reshape(pick.size, -1)
    lit = (db64 > db64.max(axis=0)[None, :] - 30.0).ravel()
    worst = int(np.argmax(ddb))
    return {"angles": int(pick.size), "samples": int(ddb.size),
            "max_abs_ddb": float(ddb.max()), "p99_abs_ddb": float(np.percentile(ddb, 99)),
            "frac_within_0.1dB": float((ddb <= 0.1).mean()),
            "max_abs_ddb_within_30dB_of_peak": float(ddb[lit].max()),
            "samples_within_30dB_of_peak": int(lit.sum()),
            "worst_sample": {"theta": float(w["theta"][pick][worst // len(w["freqs"])]),
                             "phi": float(w["phi"][pick][worst // len(w["freqs"])]),
                             "freq_ghz": float(w["freqs"][worst % len(w["freqs"])]) / 1e9,
                             "dbsm_fp64": float(b.rcs_dbsm[worst]), "dbsm_mixed": float(a.rcs_dbsm[worst])},
            "max_field_diff_rel_to_max": float(np.abs(a.field - b.field).max() / np.abs(b.field).max()),
            "stated_error": {"what": "sbr_error_bound: per-sample bound on |dBsm - dBsm_FP64| of the mixed result",
                             "max_db": float(ed.max()), "median_db": float(np.median(ed)),
                             "p99_db": float(np.percentile(ed, 99)),
                             "samples_where_bound_holds": int((ddb <= ed + 1e-9).sum()),
                             "field_bound_holds": int((np.abs(a.field - b.field) <= ef).sum()),
                             "median_bound_over_measured": float(np.median(ed / np.maximum(ddb, 1e-12))),
                             "wall_s": bound_s},
            "fp64_ms": b.device_ms, "mixed_ms": a.device_ms}


def per_angle_leg(w, sbr, scene, sp, torch, stream, stride: int, value: float) -> dict:
    """The engine in the reference's loop structure (one trace + PO launch per (angle,
    frequency), each frequency on its own grid, FP32 arithmetic) on every
    `stride`-th angle, and its fields against the batched engine's."""
    sub = slice(0, None, stride)
    pjobs = [sbr.JobSpec(w["theta"][sub], w["phi"][sub], [f], w["grid"][f], w["grid"][f], w["G"], w["max_bounces"],
                         w["R"]) for f in w["freqs"]]
    pplan = sbr.Plan(scene, pjobs, mode=sbr.MODE_PER_ANGLE, precision=sbr.PREC_FP32, stream=sp)
    pplan.execute()  # untimed warm-up
    pplan.results()
    torch.cuda.synchronize()
    pa0, pa1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pa0.record(stream)
    pplan.execute()
    pa1.record(stream)
    torch.cuda.synchronize()
    pa_ms = pa0.elapsed_time(pa1)
    per_angle_value = pplan.info["n_samples"] / (pa_ms * 1e-3)
    pres = pplan.results()
    bjob = sbr.JobSpec(w["theta"][sub], w["phi"][sub], w["freqs"], w["nx"], w["ny"], w["G"], w["max_bounces"], w["R"])
    bres = sbr.run(scene, bjob, mode=sbr.MODE_BATCHED, precision=sbr.PREC_MIXED)
    nsub, nf = len(w["theta"][sub]), len(w["freqs"])
    pf = pres.field.reshape(nf, nsub).T  # per-angle plan is frequency-major (one job per frequency)
    bf = bres.field.reshape(nsub, nf)
    same_grid = all(w["grid"][f] == w["nx"] for f in w["freqs"])
    out = {"value": per_angle_value, "unit": "samples/s", "precision": "fp32 (reference arithmetic)",
           "samples": pplan.info["n_samples"], "angles": nsub, "ms": pa_ms,
           "launches": pplan.info["launches_per_execute"], "rays_launched": pplan.info["n_rays_clipped"],
           "batched_speedup": value / per_angle_value,
           "grids": "same as batched" if same_grid else "own grid per frequency (batched: finest grid)",
           "max_field_diff_vs_batched_rel_to_max": float(np.abs(pf - bf).max() / np.abs(bf).max())}
    pplan.close()
    return out


def adjoint_leg(w, sbr, scene, job, res, info, samples, sp, torch, stream, steps) -> dict:
    """Reverse-mode gradient of mean(sigma) along the frozen hit paths (sbr_adjoint)."""
    cot = 8.0 * np.pi * res.field / res.field.size
    sbr.adjoint(scene, job, cot, precision=sbr.PREC_MIXED, stream=sp)  # warm-up
    a_ms, a_dev = [], []
    gx = None
    for _ in range(max(1, min(steps, 3))):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        gx, gf = sbr.adjoint(scene, job, cot, precision=sbr.PREC_MIXED, stream=sp)
        e1.record(stream)
        a_ms.append((time.perf_counter() - t0) * 1e3)
        torch.cuda.synchronize()
        a_dev.append(e0.elapsed_time(e1))
    return {"ms": float(np.mean(a_dev)), "samples_per_s": samples / (float(np.mean(a_dev)) * 1e-3),
            "rays_per_s": info["n_rays_clipped"] / (float(np.mean(a_dev)) * 1e-3),
            "timing": "CUDA events on the launching stream around sbr_adjoint (cotangent upload, gradient "
                      "download and the plan tables included)",
            "wall_ms": float(np.mean(a_ms)),
            "grad_norm": float(np.linalg.norm(gx)), "lit_vertices": int((np.abs(gx).sum(axis=1) > 0).sum())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="aircraft",
                    choices=["aircraft", "trihedral", "sphere", "aircraft-dev", "ellipsoid", "uneven"])
    ap.add_argument("--adjoint", action="store_true",
                    help="also time the adjoint (gradient of the mean RCS w.r.t. vertices and frequency)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--angles", type=int, default=0,
                    help="profile case: trace only this many angles, evenly spread over the sweep")
    ap.add_argument("--no-per-angle", action="store_true", help="skip the per-angle mode measurement")
    ap.add_argument("--per-angle-stride", type=int, default=8,
                    help="per-angle mode is timed on every n-th angle of the sweep")
    ap.add_argument("--first-hit", default="auto", choices=["auto", "traverse", "raster"],
                    help="first closest hit: the library's choice (default: the tile raster where a plan launches "
                         ">= 8 rays per triangle per angle), the BVH walk, or the tile raster")
    ap.add_argument("--tile-cap", type=int, default=0, help="the raster's per-tile triangle list length (0: 48)")
    ap.add_argument("--autotune", action="store_true",
                    help="let the plan time candidate work-item sizes / grid sizes on a sample first")
    ap.add_argument("--polarization", default="scalar", choices=["scalar", "hhvv"],
                    help="the reference's scalar PO term, or HH and VV fields with E-vector tracking")
    ap.add_argument("--gpu-build", action="store_true", help="build the scene's SAH tree on the GPU")
    ap.add_argument("--node-width", type=int, default=4, choices=[4, 8],
                    help="BVH node width walked by the sweep kernel (8: the opt-in 8-wide tree)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the reference's own GPU build (baseline/_ref) on the same GPU")
    ap.add_argument("--fp64-check", type=int, default=16,
                    help="compare with a full-FP64 run of the batched job on this many angles (0: skip)")
    ap.add_argument("--no-counts", action="store_true", help="skip the oracle's per-query counts (roofline)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import sagittasbr_b200 as sbr

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    if args.workload == "uneven":
        rc = run_uneven(args, torch, sbr, dist, ws, rank, local)
        if dist is not None:
            dist.destroy_process_group()
        return rc
    w = workload(args.workload)
    if args.angles > 0:
        pick = np.linspace(0, w["theta"].size - 1, args.angles).round().astype(int)
        w["theta"], w["phi"] = w["theta"][pick], w["phi"][pick]
        w["name"] += f"_subset{args.angles}"
    # a real stream: the library treats a null handle as "its own stream", so the
    # legacy default stream (handle 0) cannot be shared with torch's events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    t_scene = time.perf_counter()
    scene = sbr.Scene(w["verts"], w["tris"], device=local, gpu_build=args.gpu_build, node_width=args.node_width)
    scene_s = time.perf_counter() - t_scene
    sah_ms = scene.info()["sah_ms"]
    job = sbr.JobSpec(w["theta"], w["phi"], w["freqs"], w["nx"], w["ny"], w["G"], w["max_bounces"], w["R"])
    first_hit = {"auto": sbr.FIRST_HIT_AUTO, "raster": sbr.FIRST_HIT_RASTER,
                 "traverse": sbr.FIRST_HIT_TRAVERSE}[args.first_hit]
    pol = sbr.POL_HHVV if args.polarization == "hhvv" else sbr.POL_SCALAR
    from sagittasbr_b200.sharding import ShardedPlan
    t_plan = time.perf_counter()
    shard = ShardedPlan(scene, job, rank, ws, mode=sbr.MODE_BATCHED, precision=sbr.PREC_MIXED, stream=sp,
                        first_hit=first_hit, polarization=pol, autotune=args.autotune,
                        tile_cap=args.tile_cap) if ws > 1 else None
    plan = shard.plan if shard is not None else sbr.Plan(scene, [job], mode=sbr.MODE_BATCHED,
                                                         precision=sbr.PREC_MIXED, stream=sp, first_hit=first_hit,
                                                         polarization=pol, autotune=args.autotune,
                                                         tile_cap=args.tile_cap)
    plan_s = time.perf_counter() - t_plan
    info = plan.info if plan is not None else {"n_samples": 0, "n_rays_clipped": 0, "launches_per_execute": 0,
                                               "blocks_per_item": 0, "ctas_per_sm": 0, "h2d_bytes": 0,
                                               "d2h_bytes": 0}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def step():
        if shard is not None:
            shard.execute()
            return shard.gather(torch)
        plan.execute()
        return None

    for _ in range(args.warmup):
        flush.zero_()
        step()
    res = plan.results() if plan is not None else None
    bounces_step = res.bounces if res is not None else 0
    queries_step = res.queries if res is not None else 0
    barrier()
    clocks = Clocks(local) if rank == 0 else None
    per = []
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        merged = step()
        e1.record(stream)
        per.append((e0, e1))
    t_end.record(stream)
    barrier()
    clk = clocks.stop() if clocks else None
    total_ms = t_start.elapsed_time(t_end)
    kern_ms = float(np.mean([a.elapsed_time(b) for a, b in per]))
    ms = torch.tensor([total_ms / args.steps, kern_ms], device="cuda", dtype=torch.float64)
    cnt = torch.tensor([float(bounces_step), float(queries_step)], device="cuda", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        dist.all_reduce(cnt, op=dist.ReduceOp.SUM)
    step_ms, kern_ms = float(ms[0]), float(ms[1])
    bounces_all, queries_all = float(cnt[0]), float(cnt[1])
    samples = int(w["theta"].size) * len(w["freqs"])
    value = samples / (step_ms * 1e-3)

    # end to end through the public API, host arrays in and out: sbr_run on one GPU,
    # the sharded sweep (plan per rank + gather) under torchrun
    e2e_ms = []
    r2 = None
    for s in range(1 + max(3, min(args.steps, 5))):
        barrier()
        t0 = time.perf_counter()
        if shard is None:
            r2 = sbr.run(scene, job, mode=sbr.MODE_BATCHED, precision=sbr.PREC_MIXED, first_hit=first_hit,
                         polarization=pol, blocks_per_item=info["blocks_per_item"], tile_cap=args.tile_cap)
        else:
            e2 = ShardedPlan(scene, job, rank, ws, mode=sbr.MODE_BATCHED, precision=sbr.PREC_MIXED, stream=sp,
                             first_hit=first_hit, polarization=pol, tile_cap=args.tile_cap)
            e2.execute()
            r2 = e2.gather(torch)
            e2.close()
        if s:
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_t = torch.tensor([float(np.median(e2e_ms)), float(np.mean(e2e_ms))], device="cuda", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = samples / (float(e2e_t[0]) * 1e-3)
    if shard is None:
        assert np.array_equal(r2.field, res.field), "sbr_run and plan results differ"
    elif rank == 0:
        assert np.array_equal(r2, merged), "sharded end-to-end and plan results differ"

    # the remaining legs run on rank 0 alone, after the timed region
    per_angle = adj = fp64 = refg = cpu = counts = None
    if rank == 0 and ws == 1:
        if not args.no_per_angle:
            per_angle = per_angle_leg(w, sbr, scene, sp, torch, stream, args.per_angle_stride, value)
        if args.adjoint:
            adj = adjoint_leg(w, sbr, scene, job, res, info, samples, sp, torch, stream, args.steps)
        if args.fp64_check > 0 and pol == sbr.POL_SCALAR:
            fp64 = fp64_check_leg(w, sbr, scene, args.fp64_check)
    if dist is not None:
        dist.barrier()
    if rank != 0:
        if shard is not None:
            shard.close()
        scene.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    peak = fp32_peak_tflops(torch)
    if not args.no_ref_gpu and ws == 1 and args.angles == 0 and args.workload in REF_GPU_SAMPLES:
        refg = ref_gpu_leg(w, sbr, scene, value)
    if not args.no_cpu and ws == 1:
        c = CpuReference(w).sample(10.0)
        cpu = {"value": c["value"], "unit": "samples/s", "cores": os.cpu_count(), "kind": "reference",
               "sample": c["sample"], "mray_bounces_per_s": c["mray_bounces_per_s"], "rays_per_s": c["rays_per_s"]}
    if not args.no_counts:
        counts = oracle_counts(w)
    roof = None
    if counts is not None and queries_all > 0:
        vbox, vtri = counts["v_box"], counts["v_tri"]
        flop_q = FLOP_PER_BOX * vbox + FLOP_PER_TRI * vtri
        achieved = queries_all * flop_q / (kern_ms * 1e-3) / 1e12
        fh_name = {sbr.FIRST_HIT_RASTER: "tile raster", sbr.FIRST_HIT_TRAVERSE: "walk"}.get(info.get("first_hit"))
        dq = DRAM_BYTES_PER_QUERY.get((args.workload, fh_name))
        hbm, hbm_src = hbm_peak_gbs()
        roof = {"bound": "fp32", "achieved": achieved, "peak": peak * ws, "unit": "TFLOP/s",
                "frac": achieved / (peak * ws),
                "traffic": dq * queries_all / ws if dq is not None else None,
                "kernel": ("k_tile_bin + k_tile_hit + k_trace (persistent) + k_finalize" if fh_name == "tile raster"
                           else "k_trace (persistent) + k_finalize"),
                "flop_per_query": flop_q, "v_box": vbox, "v_tri": vtri,
                "queries_per_launch": queries_all / ws, "counts": counts,
                "peak_source": "FP32 SGEMM 8192^3 measured in this run, per GPU (no FP32 figure in the peaks file)",
                "fp32_fma_rate_at_sampled_clock": (fma_peak_tflops(torch, clk["sm_mhz"]) if clk else None),
                "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per query of a subset capture, "
                                   "x queries of a full launch") if dq is not None else None,
                "hbm_view": {"bytes_per_query": 48 * (vbox + vtri),
                             "achieved_GBs": queries_all * 48 * (vbox + vtri) / (kern_ms * 1e-3) / 1e9 / ws,
                             "peak_GBs": hbm, "peak_source": hbm_src,
                             "note": "reference-tree node+triangle bytes per GPU; mostly served from L1/L2"}}
    line = {
        "metric": "angle-freq samples/s", "value": value, "unit": "samples/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None, "dtype": "fp32 traversal + fp32-pair phase + fp64 sums",
        "data": f"synthetic (seeded {args.workload} mesh)",
        "config": config_of(w),
        "run": {"rays_launched_per_step": info["n_rays_clipped"], "mode": "batched persistent",
                "precision": "mixed", "polarization": args.polarization,
                "parallelism": (f"{ws} GPUs, cost-balanced angle shards of one sweep, fields gathered to rank 0 "
                                "inside the timed region") if ws > 1 else "1 GPU",
                "scene_build_s": scene_s, "sah_build": {"where": "gpu" if args.gpu_build else "host", "ms": sah_ms},
                "plan_s": plan_s, "autotune": bool(args.autotune), "node_width": args.node_width,
                "blocks_per_item": info["blocks_per_item"], "ctas_per_sm": info["ctas_per_sm"],
                "first_hit": {sbr.FIRST_HIT_RASTER: "tile raster", sbr.FIRST_HIT_TRAVERSE: "walk"}.get(
                    info.get("first_hit"), None), "tile_cap": args.tile_cap or 48},
        "mray_bounces_per_s": bounces_all / (step_ms * 1e-3) / 1e6,
        "closest_hit_queries_per_s": queries_all / (step_ms * 1e-3),
        "kernel_ms": kern_ms,
        "per_angle": per_angle,
        "reference_gpu": refg,
        "fp64_check": fp64,
        "adjoint": adj,
        "e2e": {"value": e2e_value, "unit": "samples/s", "h2d_bytes_per_step": info["h2d_bytes"] * ws,
                "d2h_bytes_per_step": info["d2h_bytes"] * ws, "ms_per_step": float(e2e_t[0]),
                "mean_ms_per_step": float(e2e_t[1]),
                "timing": "wall clock around " + ("sbr_run" if ws == 1 else "ShardedPlan create + execute + gather")
                          + ", median of the timed calls (mean beside it)", "calls_ms": e2e_ms},
        "gpu_launches": int(info["launches_per_execute"]) * args.steps,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    if shard is not None:
        shard.close()
    else:
        plan.close()
    scene.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
