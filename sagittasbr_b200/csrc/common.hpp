// common.hpp -- internal types shared by the host set-up and the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "sbr.h"

namespace sbr {

// ------------------------------------------------------------------ errors
// Thread-local detail message behind sbr_last_error().
void set_error(const std::string& msg);
sbr_status fail(sbr_status s, const std::string& msg);
sbr_status cuda_fail(cudaError_t e, const char* what);

#define SBR_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e__ = (call);                           \
        if (e__ != cudaSuccess) return sbr::cuda_fail(e__, #call); \
    } while (0)

// Makes an entry point leave the caller's current device as it found it: records
// the current device on construction and sets it back on every return path.
class DeviceGuard {
  public:
    DeviceGuard() {
        if (cudaGetDevice(&prev_) != cudaSuccess) prev_ = -1;
    }
    ~DeviceGuard() {
        if (prev_ >= 0) cudaSetDevice(prev_);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;

  private:
    int prev_ = -1;
};

// Zeroes one 32-bit device word before returning (a copy from pageable host memory
// completes before cudaMemcpy returns; a cudaMemset would be queued on the legacy
// stream, which the non-blocking streams the kernels run on do not wait for).
template <class T>
inline cudaError_t clear_device_word(T* d) {
    static_assert(sizeof(T) == 4, "a 32-bit word");
    const T zero = 0;
    return cudaMemcpy(d, &zero, sizeof(T), cudaMemcpyHostToDevice);
}

// Device-side error word bits (written by kernels, read after each execute).
enum : uint32_t {
    DEV_ERR_STACK = 1u,      // traversal stack would overflow (entry dropped)
    DEV_ERR_BUDGET = 2u,     // per-query iteration budget exceeded
    DEV_ERR_CANCEL = 4u,     // cancel flag observed
};

// ------------------------------------------------------------- GPU layout
// 4-wide BVH node: the boxes of up to four children in structure-of-arrays form
// (each float4 holds one plane of all four children) and their references, seven
// 16 B loads.  Child reference: >= 0 inner node index; < 0 leaf, where
// ~ref = first_triangle * 16 + count (count 1..15).  Empty slots hold a point box
// far outside any ray's reach (it never passes the slab test) and reference ~0.
struct __align__(16) GNode4 {
    float4 lox, hix, loy, hiy, loz, hiz;
    int4 child;
};
static_assert(sizeof(GNode4) == 112, "GNode4 must be 112 bytes");

// 8-wide node (opt-in, sbr_build_opts.node_width = 8): two 4-wide halves holding
// children 0-3 and 4-7, fourteen 16 B loads.  Inner child references index the
// 8-wide node array; leaves and empty slots are encoded as in GNode4.
struct __align__(16) GNode8 {
    GNode4 q[2];
};
static_assert(sizeof(GNode8) == 224, "GNode8 must be 224 bytes");

constexpr int kLeafMax = 15;
constexpr int kStackDepth = 64;     // reference uses 64 (src/cuda/rtKernels.cu:65)

// Leaf-ordered triangle: the three FP32 vertices and the unit normal
// unit(e1 x e2), e1 = v1 - v0, e2 = v2 - v0, in the w lanes (three 16 B loads).
// Vertices rather than edges: triangles sharing an edge then hold bit-identical
// copies of its end points, which the watertight test needs; Moller-Trumbore forms
// the edges in the kernel with the same FP32 subtraction the reference does.
struct __align__(16) GTri {
    float4 v0;    // v0.xyz, n.x
    float4 v1;    // v1.xyz, n.y
    float4 v2;    // v2.xyz, n.z
};

// FP64 twin of GTri used by SBR_PREC_FP64.
struct GTri64 {
    double v0[3], e1[3], e2[3], n[3];
};

struct SceneView {
    const GNode4* __restrict__ nodes;
    const GTri* __restrict__ tris;
    const GTri64* __restrict__ tris64;
    const int32_t* __restrict__ tri_id;
    const GNode8* __restrict__ nodes8;  // the 8-wide tree of the same leaves, or null
    const int32_t* __restrict__ tie;    // per slot: rank in the reference's walk order, or null
};

// --------------------------------------------------------------- plan data
// One (job, angle) of a plan.  Frames are computed on the host in FP64.
struct __align__(16) Segment {
    double dir[3];        // incidence direction (toward the launcher)
    double llc[3];        // launch corner used by this plan (reference corner at 10 G, minus shift * dir)
    double u[3], v[3];    // launcher edge vectors (length G)
    double shift;         // distance the launch plane was moved toward the scene (added back to the path)
    float llcf[3];        // FP32 launch corner
    float uf[3], vf[3];   // FP32 edge vectors
    float rdf[3];         // FP32 ray direction (-dir)
    int32_t job;          // job index
    int32_t angle;        // angle index within the job
    int32_t i0, j0;       // first ray (pixel) of the clipped rectangle
    int32_t ni, nj;       // clipped rectangle size in rays
    int32_t blocks_x;     // ray blocks across the clipped rectangle
    int32_t blocks;       // blocks in the clipped rectangle
    int32_t blocks_per_item;
    int32_t tbase;        // first-hit raster: first tile (ray block) of this segment within its chunk
    int64_t item_base;    // first work item of this segment
    int64_t sample_base;  // first output sample (angle, freq) index
    // pixel coordinates of a point P on the launcher grid: s = ps[0..2].P + ps[3],
    // t = pt[0..2].P + pt[3] (pixel (i, j) is centred at s = i, t = j)
    double ps[4], pt[4];
    int64_t zbase;        // first first-hit buffer entry of this segment within its chunk (32 tbase;
                          // entries are tile-major: tile, then lane of the 4 x 8 block)
};
// Per (job, angle) data of SBR_POL_HHVV plans: the transmit / receive unit vectors
// e_H = phi-hat = (-sin phi, cos phi, 0) and e_V = theta-hat =
// (cos theta cos phi, cos theta sin phi, -sin theta), and the distance of the
// reference launch plane (the reference's corner at 10 G) from the origin along the
// incidence direction, which the exit path is measured back to.
struct SegPol {
    double eh[3], ev[3];
    double plane;
    double pad;
};

struct JobConst {
    int32_t nx, ny;
    int32_t n_freqs;
    int32_t max_bounces;
    int32_t freq_base;    // index of this job's first frequency in the frequency table
    int32_t scene;        // index of the job's scene in a multi-scene plan (0 otherwise)
    double inv_nx, inv_ny;
    double refl;          // reflection coefficient R
    float reflf;
    float pad2;
};

// Per frequency: k, the PO scale k*A/(4 pi) (ray area of the owning job), the
// fixed-point quantum of the field accumulators, the phase of a unit path length
// of the scalar term in turns (2 k / (2 pi)), and FP32 copies used by the
// reference FP32 arithmetic.
struct FreqConst {
    double k;
    double scale;         // k * rayArea / (4 pi)
    double quantum;       // field value of one accumulator unit
    double inv_quantum;
    double turns;         // k / pi
    float kf;
    float scalef;
    float turns_hi, turns_lo;  // k / pi as an unevaluated FP32 pair (hi + lo)
};

struct ItemStats {
    uint32_t rays, hit_rays, bounces, queries;
};

// Rays are handed out in blocks of 4 x 8 pixels, 4 along the launcher's u axis and
// 8 along v (one warp's worth of spatially adjacent, parallel rays); a work item
// is a run of consecutive blocks of one segment, owned by one warp.  Measured on
// B200 against 8 x 4, 16 x 2 and 2 x 16: 4 x 8 traced 1.5 % (trihedral) to 5 %
// (SH ellipsoid) faster than 8 x 4, the others slower.
constexpr int kBlockW = 4;
constexpr int kBlockH = 8;
static_assert(kBlockW * kBlockH == 32, "a ray block is one warp");
constexpr int kCtaThreads = 128;     // 4 independent warps per CTA
constexpr int kAccReplicas = 8;      // copies of each accumulator (spreads same-address atomics)

}  // namespace sbr
