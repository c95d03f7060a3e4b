// plan.hpp -- the opaque handles behind sbr_scene and sbr_plan.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "common.hpp"

struct sbr_scene {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    int64_t ntris = 0;
    double model_scale = 1.0;
    double aabb_lo[3] = {0, 0, 0}, aabb_hi[3] = {0, 0, 0};  // conservative, FP64
    // host copies kept for the FP64 upload and diagnostics
    std::vector<float> xyz;          // caller vertices (unscaled)
    std::vector<uint32_t> idx;
    std::vector<int32_t> order;      // leaf slot -> caller triangle index
    // device
    sbr::GNode4* d_nodes = nullptr;
    int64_t n_gnodes = 0;
    sbr::GNode8* d_nodes8 = nullptr;  // node_width 8: the same leaves under 8-wide nodes
    int64_t n_gnodes8 = 0;
    int64_t n_bin_nodes = 0;
    sbr::GTri* d_tris = nullptr;
    sbr::GTri64* d_tris64 = nullptr;
    int32_t* d_tri_id = nullptr;
    int32_t* d_tie = nullptr;        // exact-tie ranks (coincident faces of opposite winding), or null
    float* d_xyz = nullptr;          // caller vertices and triangles, uploaded for the adjoint
    uint32_t* d_idx = nullptr;
    uint32_t* d_err = nullptr;
    int32_t* d_cancel = nullptr;     // device word polled by the kernels
    int32_t* h_flag_vals = nullptr;  // pinned {1, 0}: sources of the async flag copies
    cudaStream_t cancel_stream = nullptr;
    int depth = 0;
    double build_ms = 0.0;
    double sah_ms = 0.0;
    // refit: 4-wide node indices grouped by depth (offsets per depth), their device
    // copy, and the per-triangle box scratch of a refit
    std::vector<int32_t> refit_nodes;
    std::vector<int32_t> refit_level_off;
    int32_t* d_refit_nodes = nullptr;
    float* d_tri_box = nullptr;
    int64_t device_bytes = 0;

    sbr::SceneView view() const { return sbr::SceneView{d_nodes, d_tris, d_tris64, d_tri_id, d_nodes8, d_tie}; }
};

struct sbr_plan {
    sbr_scene* scene = nullptr;
    int mode = SBR_MODE_BATCHED;
    int prec = SBR_PREC_MIXED;
    int pol = SBR_POL_SCALAR;
    int use_graph = 0;
    int ctas_per_sm = 0;
    int blocks_per_item = 0;
    int node_width = 4;                      // tree the mixed scalar sweep walks
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    sbr::SceneView scene_view{};
    bool multi = false;                      // jobs trace different scenes (JobConst::scene)
    std::vector<sbr::SceneView> scene_views; // multi-scene plans: one per scene
    sbr::SceneView* d_scenes = nullptr;

    std::vector<sbr::Segment> segs;
    std::vector<int64_t> seg_base;     // [n_segs + 1] first item of each segment
    std::vector<sbr::JobConst> jobs;
    std::vector<sbr::FreqConst> freqs;
    std::vector<double> quantum;       // per sample and polarisation
    std::vector<sbr::SegPol> segpol;   // per segment (SBR_POL_HHVV)
    int n_pol = 1;
    int64_t n_segs = 0, n_items = 0, n_samples = 0;
    int64_t n_rays_clipped = 0, n_rays_grid = 0;
    int k_max = 1;
    int persistent_grid = 0;
    int launches = 0;

    // device
    sbr::Segment* d_segs = nullptr;
    int64_t* d_seg_base = nullptr;
    sbr::JobConst* d_jobs = nullptr;
    sbr::FreqConst* d_freqs = nullptr;
    double* d_quantum = nullptr;
    sbr::SegPol* d_segpol = nullptr;
    unsigned long long* d_acc = nullptr;
    unsigned long long* d_acc_stats = nullptr;
    double* d_field = nullptr;
    unsigned long long* d_stats = nullptr;
    unsigned long long* d_queue = nullptr;
    uint32_t* d_err = nullptr;
    const volatile int32_t* d_cancel = nullptr;
    int64_t device_bytes = 0;

    // first-hit rasterisation: segments are processed in chunks whose first-hit
    // buffers fit `d_zbuf`; each chunk = tile binning + tile raster + trace launch
    struct Chunk {
        int64_t seg_begin, seg_end, item_begin, item_end, zcount, tiles;
    };
    bool raster = false;
    std::vector<Chunk> chunks;
    unsigned long long* d_zbuf = nullptr;
    int64_t zbuf_elems = 0;
    int64_t tiles_max = 0;              // tiles of the largest chunk
    uint32_t tile_cap = 0;              // list entries per tile (longer lists walk)
    uint32_t* d_tile_cnt = nullptr;     // [tiles_max]
    int32_t* d_tile_list = nullptr;     // [tiles_max * tile_cap]

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool executed = false;
};

namespace sbr {

// Receives the host tables of a sweep as build_tables produces them; a sink
// returns false when it has no room left.
struct TableSink {
    virtual ~TableSink() = default;
    virtual bool job(const JobConst& j) = 0;
    virtual bool freq(const FreqConst& f) = 0;
    // one (job, angle) segment, the first item of the next segment, and the job's
    // per-frequency accumulator units (one per output sample of this segment)
    virtual bool segment(const Segment& g, int64_t next_item, const double* quantum, int n_freqs) = 0;
};

struct TableTotals {
    int64_t n_segs = 0, n_items = 0, n_samples = 0, n_rays_clipped = 0, n_rays_grid = 0;
    int k_max = 1;
};

// Argument checks shared by every sweep entry point.
sbr_status validate_run(const sbr_scene* s, const sbr_job* jobs, size_t n_jobs, const sbr_run_opts& o);
// Launcher frames, aperture clipping, work items and fixed-point units of a sweep.
// Job j is clipped against the bounds of job_scene[j] (an index into scenes) when
// job_scene is given, else every job uses scenes[0].
sbr_status build_tables(const sbr_scene* const* scenes, const int32_t* job_scene, const sbr_job* jobs,
                        size_t n_jobs, const sbr_run_opts& o, TableSink& sink, TableTotals& tot);

sbr_status plan_launch(sbr_plan* pl, bool records, sbr_ray_record* d_records);

sbr_status fill_records(sbr_ray_record* d, long long n, cudaStream_t st);
// Traces the listed rays (angle index, i, j; checked by the caller) of a one-job plan.
sbr_status trace_list_launch(sbr_plan* pl, const int32_t* d_rays, long long n, sbr_ray_record* d_out);
int max_freqs_per_job();
sbr_status ensure_fp64(sbr_scene* s);
sbr_status ensure_adjoint_data(sbr_scene* s);
}  // namespace sbr
