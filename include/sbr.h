/* sbr.h -- C ABI of libsbr, the B200-native shooting-and-bouncing-rays (SBR)
 * monostatic RCS engine.
 *
 * This boundary replaces SagittaSBR's device seam
 *
 *     sweepResults runSweep(const simulationConfig&, deviceBuffers&,
 *                           const bvhGpuData&, std::ostream&)      include/sim/sweep.hpp:15-16
 *
 * and the set-up that feeds it in runRcsApp (src/app/rtRcsEntry.cu:115-196:
 * de-indexing, model scale, buildBvh, cudaMalloc/cudaMemcpy of triangles and
 * nodes, allocateDeviceBuffers).  Plain pointers and sizes only; every call
 * returns a status (the reference calls cudaDeviceReset + exit(1) on any CUDA
 * error, src/cuda/cudaUtils.cu:6-14; this library never exits).
 *
 * Threading: a scene or plan handle is used by one host thread at a time.
 * Device memory belongs to the scene / plan that allocated it.
 */
#ifndef SBR_H
#define SBR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SBR_ABI_VERSION 3  /* 2: sbr_config.error_bound, sbr_build_opts / sbr_run_opts / sbr_plan_info.node_width;
                              3: SBR_FIRST_HIT_AUTO (0, the default), sbr_run_opts.tile_cap,
                                 sbr_plan_info.first_hit */

/* ------------------------------------------------------------------ status */
typedef int32_t sbr_status;
#define SBR_OK 0
#define SBR_ERR_INVALID_ARG 1   /* null pointer, bad size, bad enum           */
#define SBR_ERR_EMPTY_MESH 2    /* no triangles (rtRcsEntry.cu:109-113)       */
#define SBR_ERR_BAD_INDEX 3     /* vertex index out of range (:126-130)       */
#define SBR_ERR_NONFINITE 4     /* NaN/Inf vertex or parameter                */
#define SBR_ERR_TOO_LARGE 5     /* grid or mesh beyond the supported size     */
#define SBR_ERR_CUDA 6          /* CUDA runtime error (message in last_error) */
#define SBR_ERR_OOM 7           /* device allocation failed                   */
#define SBR_ERR_NO_DEVICE 8     /* no usable sm_100 device                    */
#define SBR_ERR_STACK 9         /* traversal stack overflow reported by GPU   */
#define SBR_ERR_TIMEOUT 10      /* iteration budget exceeded on the GPU       */
#define SBR_ERR_CANCELLED 11    /* sbr_scene_cancel() observed by the kernel  */
#define SBR_ERR_IO 12           /* file could not be read / written           */
#define SBR_ERR_PARSE 13        /* malformed model / config file             */
#define SBR_ERR_UNSUPPORTED 14  /* option or combination not supported          */

/* Short name of a status code (static string). */
const char* sbr_status_str(sbr_status s);
/* Detail message of the last failing call on this host thread (static per thread). */
const char* sbr_last_error(void);
int32_t sbr_abi_version(void);

/* ------------------------------------------------------------------- scene */
typedef struct sbr_scene sbr_scene;

typedef struct sbr_build_opts {
    double model_scale;   /* vertices are multiplied by this (--model-scale, rtRcsEntry.cu:137-145); 0 -> 1 */
    int32_t device;       /* CUDA device ordinal; -1 -> current device */
    int32_t leaf_size;    /* max triangles per BVH leaf; 0 -> 3 (the reference's builder uses 4,
                             bvhBuilder.hpp:14; 3 traces faster with 4-wide nodes) */
    int32_t bin_count;    /* SAH bins; 0 -> 16 (bvhBuilder.hpp:15) */
    int32_t n_threads;    /* host threads for the build; 0 -> all */
    int32_t want_fp64;    /* also upload FP64 triangles (needed by SBR_PREC_FP64); -1 -> lazily */
    int32_t gpu_build;    /* 1: build the binary SAH tree on the GPU (same tree as the host build;
                             triangles inside a leaf may be ordered differently) */
    int32_t node_width;   /* 0 or 4: 4-wide nodes (default); 8: the mixed-precision scalar sweep
                             walks 8-wide nodes built over the same leaves (the other kernels keep
                             the 4-wide tree; the same closest hits either way) */
    int32_t reserved[1];
} sbr_build_opts;

typedef struct sbr_scene_info {
    int64_t n_triangles;
    int64_t n_nodes_bin;      /* binary SAH nodes */
    int64_t n_nodes_gpu;      /* nodes of the traversal layout in HBM */
    int64_t device_bytes;     /* scene bytes resident on the device */
    double aabb_lo[3];
    double aabb_hi[3];
    double build_ms;          /* scene set-up time (BVH build, layout, upload) */
    int32_t device;
    int32_t bvh_depth;
    double sah_ms;            /* of which the binary SAH build (host threads or GPU) */
} sbr_scene_info;

/* Copies the indexed triangle mesh (xyz: nverts*3 floats, tri_idx: ntris*3
 * indices), builds the BVH (SAH tree on host threads, or on the GPU with
 * opts->gpu_build) and uploads it.  The caller keeps its buffers.  Replaces
 * rtRcsEntry.cu:115-196.  A mesh that holds a triangle twice with opposite
 * windings also gets each triangle's rank in the reference's closest-hit walk
 * (one more host SAH build, 4 bytes per triangle on the device): on an exact tie
 * the sweep keeps the triangle that walk keeps (src/cuda/rtKernels.cu:36). */
sbr_status sbr_scene_create(const float* xyz, size_t nverts, const uint32_t* tri_idx, size_t ntris,
                            const sbr_build_opts* opts, sbr_scene** out);
sbr_status sbr_scene_destroy(sbr_scene* scene);
sbr_status sbr_scene_info_get(const sbr_scene* scene, sbr_scene_info* out);
/* Asks running kernels of this scene to stop at their next work item
 * (they return SBR_ERR_CANCELLED); sbr_scene_reset_cancel clears it. */
sbr_status sbr_scene_cancel(sbr_scene* scene);
sbr_status sbr_scene_reset_cancel(sbr_scene* scene);
/* New coordinates for the scene's vertices (same count, same triangles), with the
 * BVH refitted on the GPU: triangle data and every node box are recomputed for the
 * new positions while the tree topology is kept, instead of a full rebuild
 * (src/scene/bvhBuilder.cpp:315-360) -- for shape optimisation, where every
 * gradient step moves the vertices a little (traversal slows down as the
 * deformation grows; create a new scene then).  Plans created before the update
 * keep their launcher tables (aperture clipping, launch-plane placement): create
 * plans after it.  An opt-in 8-wide tree (node_width 8) is released, not refitted.
 * No counterpart in the reference. */
sbr_status sbr_scene_update_vertices(sbr_scene* scene, const float* xyz, size_t nverts);

/* --------------------------------------------------------------------- job */
/* One job = a list of incidence angles traced on one ray grid, with a set of
 * frequencies that share that grid.  The reference runs one (angle, frequency)
 * per iteration with nx*ny rays over a square of side grid_size placed
 * 10*grid_size from the origin (src/app/sweep.cu:50-55,336-397). */
typedef struct sbr_job {
    const double* theta_deg;  /* [n_angles] */
    const double* phi_deg;    /* [n_angles] */
    int64_t n_angles;
    const double* freq_hz;    /* [n_freqs] */
    int64_t n_freqs;
    int32_t nx, ny;           /* ray grid (n_x, n_y) */
    double grid_size;         /* launcher side G in metres (grid_size) */
    int32_t max_bounces;      /* max_bounces */
    double reflection_const;  /* reflection_const (R per bounce, 1 = PEC) */
} sbr_job;

#define SBR_MODE_BATCHED 0    /* one persistent launch drains every (job, angle, tile) item; all
                                 frequencies of a job come from one trace */
#define SBR_MODE_PER_ANGLE 1  /* the reference's loop: one trace + PO launch per (angle, frequency) */

#define SBR_PREC_MIXED 0      /* FP32 traversal, FP64 path length, FP32-pair phase reduction, FP64 field sums */
#define SBR_PREC_FP32 1       /* the reference FP32 build's arithmetic (launch plane at 10 G, FP32 phase) */
#define SBR_PREC_FP64 2       /* everything in FP64 (the reference USE_DOUBLE build's arithmetic) */

/* How the first closest hit of each ray is found.  Primary rays of one angle are
 * parallel and start on the launcher grid, so their first hits form an
 * orthographic z-buffer: RASTER tests every triangle against the pixels its
 * projection covers (same Moller-Trumbore arithmetic) and keeps the nearest per
 * pixel; later bounces always walk the BVH.  RASTER applies to batched FP32 /
 * mixed runs (per-angle and FP64 runs always walk).  Measured on B200 it costs
 * about as much as the walk it replaces for coherent ray tubes, so the default
 * walks. */
#define SBR_FIRST_HIT_AUTO 0      /* (default) the raster where a plan launches, per angle, at least
                                     8 rays per triangle of its scene; the walk otherwise */
#define SBR_FIRST_HIT_RASTER 1    /* first hits from the tile-binned orthographic raster (batched
                                     mixed-precision single-scene plans; others walk) */
#define SBR_FIRST_HIT_TRAVERSE 2  /* walk the BVH for every query */

/* Polarisation.  SCALAR is the reference's PO term (poKernels.cu:81-109; HH == VV).
 * HHVV (no counterpart in the reference; SBR_PREC_MIXED or SBR_PREC_FP64, at most
 * 64 frequencies per job) tracks the HH (phi-hat) and VV (theta-hat) incident
 * fields through every PEC reflection, E <- 2 (n.E) n - E, and gives each exit
 * ray the scalar gate (cos = n.(-d_last) > 0) with the co-polarised amplitude
 * 2 R^n e.(n x (d_last x E_last)) -- the PO surface current on the last surface
 * projected on the receive polarisation, equal to the scalar 2 cos R^n for a
 * single bounce -- and the physical path launch plane -> exit point -> launch
 * plane instead of the scalar term's 2 * path (so multi-bounce returns add in
 * phase).  Fields come per (sample, HH / VV). */
#define SBR_POL_SCALAR 0
#define SBR_POL_HHVV 1

typedef struct sbr_run_opts {
    int32_t mode;             /* SBR_MODE_* */
    int32_t precision;        /* SBR_PREC_* */
    int32_t polarization;     /* SBR_POL_* */
    int32_t use_graph;        /* capture plan execution in a CUDA graph (batched mode) */
    void* stream;             /* cudaStream_t to launch on; NULL -> the scene's own stream */
    int32_t ctas_per_sm;      /* persistent grid size per SM; 0 -> occupancy-derived */
    int32_t first_hit;        /* SBR_FIRST_HIT_* */
    int32_t blocks_per_item;  /* 32-ray blocks (4 x 8) per work item; 0 -> automatic (batched: blocks / 1024
                                 clamped to 1..8 per angle, per-angle mode: 1) */
    int32_t autotune;         /* 1: sbr_plan_create times candidate (blocks_per_item, ctas_per_sm)
                                 settings -- and both tree widths when the scene holds an 8-wide
                                 tree -- on a sample of the plan's angles and keeps the fastest
                                 (batched mode; adds about 20 short launches to plan creation) */
    int32_t node_width;       /* tree the mixed-precision scalar sweep walks: 0 -> the scene's widest
                                 (8 when built with sbr_build_opts.node_width = 8), 4, or 8 */
    int32_t tile_cap;         /* SBR_FIRST_HIT_RASTER: longest triangle list a 4 x 8 ray tile tests
                                 (the rays of longer tiles walk the tree); 0 -> 48, at most 1024 */
    int32_t reserved[2];
} sbr_run_opts;

/* Results for every (job, angle, frequency[, polarization]) in job order, then
 * angle order, then frequency order (then HH, VV).  Each array may be NULL. */
typedef struct sbr_result {
    double* field;            /* [n_samples * n_pol * 2]: re, im of the scattered field sum */
    double* sigma_m2;         /* [n_samples * n_pol]: 4*pi*|field|^2 (sweep.cu:228-230) */
    double* rcs_dbsm;         /* [n_samples * n_pol]: 10*log10(max(sigma, 1e-10)) (sweep.cu:231) */
    uint64_t* stats;          /* [n_job_angles * 4]: rays, hit rays, bounces, closest-hit queries */
    double device_ms;         /* out: device time of the trace + reduce launches */
} sbr_result;

/* Plans hold the per-angle launcher frames, the work-item table and the device
 * result buffers; executing a plan touches no host memory. */
typedef struct sbr_plan sbr_plan;

typedef struct sbr_plan_info {
    int64_t n_samples;        /* sum over jobs of n_angles * n_freqs */
    int64_t n_job_angles;     /* sum over jobs of n_angles */
    int64_t n_items;          /* work items (ray tiles after aperture clipping) */
    int64_t n_rays_clipped;   /* rays actually launched (inside the projected AABB) */
    int64_t n_rays_grid;      /* sum of nx*ny over job angles */
    int32_t n_pol;
    int32_t launches_per_execute; /* kernels launched by one sbr_plan_execute */
    int64_t device_bytes;
    int64_t h2d_bytes;        /* bytes sbr_plan_create copies host -> device */
    int64_t d2h_bytes;        /* bytes sbr_plan_results copies device -> host (field, stats, error word) */
    int32_t blocks_per_item;  /* the plan's setting (0: automatic per angle) */
    int32_t ctas_per_sm;      /* persistent CTAs per SM of the trace launches */
    int32_t node_width;       /* tree width the plan's mixed scalar sweep walks (4 or 8) */
    int32_t first_hit;        /* how the plan finds first hits: SBR_FIRST_HIT_RASTER or _TRAVERSE */
} sbr_plan_info;

sbr_status sbr_plan_create(sbr_scene* scene, const sbr_job* jobs, size_t n_jobs, const sbr_run_opts* opts,
                           sbr_plan** out);
/* A plan whose jobs trace different meshes: job j traces scenes[job_scene[j]].
 * All scenes live on one device and must outlive the plan; every job of every
 * scene is drained by the same persistent launch.  Errors and the cancel flag
 * are those of scenes[0]; the first-hit raster is not used.  No counterpart in
 * the reference (one mesh per process). */
sbr_status sbr_plan_create_multi(sbr_scene* const* scenes, size_t n_scenes, const int32_t* job_scene,
                                 const sbr_job* jobs, size_t n_jobs, const sbr_run_opts* opts, sbr_plan** out);
/* Launches the plan on opts->stream (or the scene stream); asynchronous. */
sbr_status sbr_plan_execute(sbr_plan* plan);
/* Waits for the plan and copies results to host arrays (any may be NULL). */
sbr_status sbr_plan_results(sbr_plan* plan, sbr_result* out);
/* Device pointers of the plan's result arrays (valid until destroy). */
sbr_status sbr_plan_device_results(sbr_plan* plan, const double** d_field, const uint64_t** d_stats);
sbr_status sbr_plan_info_get(const sbr_plan* plan, sbr_plan_info* out);
sbr_status sbr_plan_destroy(sbr_plan* plan);

/* One call: plan, execute, copy results to host, release.  Host arrays in, host
 * arrays out.  Replaces runSweep's loop (src/app/sweep.cu:332-441). */
sbr_status sbr_run(sbr_scene* scene, const sbr_job* jobs, size_t n_jobs, sbr_result* out,
                   const sbr_run_opts* opts);

/* ----------------------------------------------------- stated error vs FP64 */
/* No counterpart in the reference (it has no mixed-precision mode).
 *
 * The error, per sample, of a SBR_PREC_MIXED result of `jobs` against the
 * SBR_PREC_FP64 result of the same jobs.  A second pass traces the same rays with
 * the mixed arithmetic while carrying FP32 error bounds along each ray (origin and
 * direction rounding, per-bounce drift of the hit point, path length and normal
 * errors).  Rays whose hit decisions lie within that uncertainty of flipping (an
 * edge within reach of the ray, |det| near its 1e-6 threshold, t near tMin or tied
 * with another hit) or whose phase uncertainty exceeds 0.05 rad are re-traced with
 * the FP64 sweep's own arithmetic and their exact difference is summed; the other
 * rays differ by rounding only: the part of those errors that is the same for all
 * rays seeing the same geometry the same way (the systematic rounding of the hit
 * distance, the sine / cosine approximation) is bounded coherently, as a fraction
 * of |field|, the rest (independent from ray to ray, and the FP32 partial sums of
 * each 4x8 ray block) by a probabilistic rounding-error bound exceeded with
 * probability below 6e-8.
 *   field     [n_samples * 2] in: the mixed-precision fields sbr_run returned.
 *   err_field [n_samples] out (may be NULL): stated |field - field_FP64|.
 *   err_db    [n_samples] out (may be NULL): the |dBsm - dBsm_FP64| it implies (dBsm
 *             floored at -100 as the reference does: a stated error above |field|
 *             gives the distance to that floor).
 * The pass costs about as much as the sweep plus an FP64 trace of the re-traced
 * rays (FP64 triangles are uploaded on first use).  opts: precision must be
 * SBR_PREC_MIXED, polarization SBR_POL_SCALAR; the mode is ignored. */
sbr_status sbr_error_bound(sbr_scene* scene, const sbr_job* jobs, size_t n_jobs, const sbr_run_opts* opts,
                           const double* field, double* err_field, double* err_db);

/* ------------------------------------------------------------- diagnostics */
#define SBR_MAX_REC 16
/* Per-ray record: the reference's hit buffers (include/app/deviceBuffers.hpp:6-15)
 * plus the triangle ids of the first hits (index in the caller's mesh). */
typedef struct sbr_ray_record {
    int32_t count;            /* hitCount */
    int32_t flags;            /* bit 0: ray launched (inside the clipped aperture) */
    double dist;              /* hitDist, summed from the reference launcher plane */
    float normal[3];          /* last hit normal */
    float lastdir[3];         /* incoming direction at the last hit */
    int32_t tri[SBR_MAX_REC]; /* hit triangle ids, -1 padded */
} sbr_ray_record;

/* Traces every ray of every angle of one job and writes nx*ny records per angle
 * (angle-major, row-major j*nx + i) to the host array `out`. */
sbr_status sbr_trace_records(sbr_scene* scene, const sbr_job* job, const sbr_run_opts* opts,
                             sbr_ray_record* out);

/* Traces only the listed rays of one job, rays[3k .. 3k+2] = (angle index, i, j),
 * with the sweep's own walk and arithmetic, and writes one record per listed ray to
 * the host array `out` -- for per-ray checks on grids too large to record whole
 * (no counterpart in the reference).  A listed ray outside the job's angles or grid
 * returns SBR_ERR_INVALID_ARG before anything runs. */
sbr_status sbr_trace_ray_list(sbr_scene* scene, const sbr_job* job, const sbr_run_opts* opts, const int32_t* rays,
                              size_t n_rays, sbr_ray_record* out);

/* ----------------------------------------------------------------- adjoint */
/* No counterpart in the reference (its sweep is not differentiable).
 *
 * Reverse-mode gradient of the scalar field sweep of `jobs` along the frozen hit
 * paths: every ray is re-traced with the precision's own closest-hit walk, the
 * path through the hit triangles is re-evaluated and differentiated in FP64, and
 * hit / miss decisions and the cos > 0 gate are held fixed.
 *   cot       [n_samples * 2]: complex cotangent g of every sample's field S, so
 *             that dLoss = sum_s Re(conj(g_s) dS_s); for Loss = sum_s w_s sigma_s
 *             it is g_s = 8 pi w_s S_s.
 *   grad_xyz  [nverts * 3] out (may be NULL): dLoss / d(caller vertex coordinates)
 *             (the unscaled xyz given to sbr_scene_create).
 *   grad_freq [n_samples] out (may be NULL): dLoss / d(frequency in Hz) of each
 *             sample's own term.
 * Scalar polarisation only; at most 16 bounces and 128 frequencies per job; the
 * mode option is ignored (one persistent launch).  Gradients are summed with FP64
 * atomics, so their last bits vary from run to run. */
sbr_status sbr_adjoint(sbr_scene* scene, const sbr_job* jobs, size_t n_jobs, const sbr_run_opts* opts,
                       const double* cot, double* grad_xyz, double* grad_freq);

/* ---------------------------------------------------- allocation-free sweep */
/* No counterpart in the reference.
 *
 * sbr_run_noalloc traces one job exactly like sbr_run (batched mode) but never
 * allocates or frees device memory.  It is meant for callers that cannot call
 * cudaMalloc while they run: programs that work inside a fixed device-memory
 * budget handed out at start-up (a memory pool or caching allocator that already
 * owns the free HBM, so a fresh allocation fails or fragments it), and programs
 * whose other streams must not be stalled by the device-wide synchronisation
 * that cudaFree (and often cudaMalloc) performs.
 *
 * The sweep's scratch -- launcher frames, work-item table, fixed-point field
 * accumulators and work-queue head -- lives in one statically sized device array
 * inside libsbr (SBR_NOALLOC_SCRATCH_BYTES, held by every GPU that loads the
 * library until the process exits).  The caller passes the scene and the device
 * output arrays: d_field [n_angles * n_freqs * 2] doubles (re, im) and, if not
 * NULL, d_stats [n_angles * 4] uint64 (rays, hit rays, bounces, queries).
 *
 * Limits: one job, at most SBR_NOALLOC_MAX_ANGLES angles and
 * SBR_NOALLOC_MAX_SAMPLES angle-frequency samples per call; larger requests return
 * SBR_ERR_TOO_LARGE.  SBR_PREC_FP64 needs a scene created with want_fp64 = 1
 * (uploading FP64 triangles later would allocate); SBR_MODE_PER_ANGLE returns
 * SBR_ERR_UNSUPPORTED.
 * Set-up: the first call on a device looks up the device address of the array
 * (cudaGetSymbolAddress) with that device current; make that first call before
 * any stream capture.  The address is kept for the life of the process: a program
 * that resets the device (cudaDeviceReset) must not call sbr_run_noalloc afterwards.
 * Sharing: every call on a device uses the same array, which keeps the previous
 * call's contents; each call clears the accumulators and queue it needs.  Calls
 * whose GPU work overlapped would race on the array and corrupt each other's
 * results, so the library serialises calls (one lock per process) and each call,
 * on success and on error alike, returns only after its stream has finished the
 * work it queued; on success it returns the device error status. */
#define SBR_NOALLOC_MAX_ANGLES 1024
#define SBR_NOALLOC_MAX_SAMPLES 4096
#define SBR_NOALLOC_SCRATCH_BYTES (448u * 1024u)
sbr_status sbr_run_noalloc(sbr_scene* scene, const sbr_job* job, double* d_field, uint64_t* d_stats,
                           const sbr_run_opts* opts);

/* --------------------------------------------------------- entry surface */
/* config.txt keys and defaults of include/app/config.hpp:8-25. */
typedef struct sbr_config {
    double phi_start, phi_end;
    int32_t phi_samples;
    double theta_start, theta_end;
    int32_t theta_samples;
    double grid_size;
    int32_t nx, ny;
    int32_t tpb_x, tpb_y;     /* parsed, unused (as in the reference) */
    int32_t max_bounces;
    double reflection_const;
    double freq;
    int32_t show_info_gpu;
    int32_t show_hit_stats;
    double model_scale;
    char model_path[4096];
    int32_t freq_source;      /* 0 default, 1 config file, 2 command line */
    /* optional keys of this engine (absent from reference configs, which keep the defaults) */
    int32_t precision;        /* key "precision": SBR_PREC_* (default SBR_PREC_MIXED) */
    int32_t mode;             /* key "engine_mode": SBR_MODE_* (default SBR_MODE_BATCHED) */
    int32_t csv_digits;       /* key "csv_digits" or flag --full-precision (17): significant digits
                                 of the rcs_results.csv rows; 0 -> 6, the reference's default
                                 ostream formatting */
    int32_t error_bound;      /* key "error_bound": 1 -> RT-RCS states each row's bound on
                                 |dBsm - dBsm_FP64| (sbr_error_bound) in a fifth column
                                 rcs_err_db (mixed precision); 0 (default) -> the reference layout */
} sbr_config;

/* loadConfig (src/app/config.cpp:39-155): reads `default_path` (or --config),
 * applies --model, --model-scale and the first bare argument as frequency.
 * Never exits: a missing file keeps defaults; a flag without value returns
 * SBR_ERR_INVALID_ARG.  Warnings go to stderr as in the reference. */
sbr_status sbr_config_load(const char* default_path, int argc, const char* const* argv, sbr_config* out);
/* theta-major angle grid of src/app/sweep.cu:336-347 (n = theta_samples*phi_samples). */
sbr_status sbr_config_angles(const sbr_config* cfg, double* theta_deg, double* phi_deg);
/* OBJ reader (v / f records; polygons fan-triangulated).  *xyz and *tri_idx are
 * allocated with malloc; release with sbr_free. */
sbr_status sbr_load_obj(const char* path, float** xyz, size_t* nverts, uint32_t** tri_idx, size_t* ntris);
/* glTF 2.0 reader (.gltf with external or base64 data: buffers, binary .glb), as the
 * reference reads it through tinygltf (src/modelLoader.cpp:286-413): every TRIANGLES
 * primitive of every mesh in file order, FLOAT POSITION accessors, u8 / u16 / u32
 * indices (none: vertices in order), node transforms not applied.  Outputs as
 * sbr_load_obj. */
sbr_status sbr_load_gltf(const char* path, float** xyz, size_t* nverts, uint32_t** tri_idx, size_t* ntris);
/* loadModel (src/modelLoader.cpp:421-450): .obj, .gltf or .glb by extension, else
 * SBR_ERR_UNSUPPORTED. */
sbr_status sbr_load_model(const char* path, float** xyz, size_t* nverts, uint32_t** tri_idx, size_t* ntris);
void sbr_free(void* p);
/* Writes rcs_results.csv in the reference layout (rtRcsEntry.cu:298-303, sweep.cu:540-544);
 * rows with cfg->csv_digits significant digits (0: 6, as the reference; 17 round-trips a
 * double).  The header lines keep the reference's formatting. */
sbr_status sbr_write_csv(const char* path, const sbr_config* cfg, const double* theta_deg, const double* phi_deg,
                         const double* sigma_m2, const double* rcs_dbsm, int64_t n);
/* sbr_write_csv with a fifth column rcs_err_db (header theta,phi,rcs_m2,rcs_dbsm,rcs_err_db):
 * each row's stated bound on |dBsm - dBsm_FP64| from sbr_error_bound. */
sbr_status sbr_write_csv_err(const char* path, const sbr_config* cfg, const double* theta_deg,
                             const double* phi_deg, const double* sigma_m2, const double* rcs_dbsm,
                             const double* err_db, int64_t n);

#ifdef __cplusplus
}
#endif
#endif /* SBR_H */
