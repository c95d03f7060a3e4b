// refit.cu -- sbr_scene_update_vertices: new vertex coordinates for an existing
// scene, with its BVH refitted on the GPU.  The tree topology (which triangles
// share a leaf, which nodes share a parent) is kept and every box is recomputed
// for the new positions, replacing a full rebuild (src/scene/bvhBuilder.cpp:315-360)
// between the steps of a shape optimisation, where each gradient step moves the
// vertices a little.
//
//   k_refit_tris   one thread per leaf slot: the triangle's FP32 data (v0, v1, v2,
//                  unit normal) in exactly the host set-up's arithmetic (scene.cpp:
//                  products and sums rounded one by one, no contraction), its FP64
//                  twin when the scene has one, and its conservative box (covering
//                  the FP32 and the outward-rounded FP64 vertices);
//   k_refit_level  one thread per 4-wide node of one depth, deepest depth first:
//                  each child slot's box becomes the union of its leaf's triangle
//                  boxes or of its child node's slot boxes.
#include <algorithm>
#include <cmath>
#include <vector>

#include "plan.hpp"

namespace sbr {
namespace {

constexpr unsigned kRefitThreads = 256;

__global__ void k_refit_tris(const float* __restrict__ xyz, const uint32_t* __restrict__ idx,
                             const int32_t* __restrict__ tri_id, int64_t ntris, float sc32, double sc, GTri* tris,
                             GTri64* tris64, float* box) {
    const int64_t slot = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (slot >= ntris) return;
    const int64_t t = tri_id[slot];
    float p[3][3];
    double q[3][3];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < 3; ++c) {
        const uint32_t v = idx[3 * t + c];
        for (int a = 0; a < 3; ++a) {
            const float x = xyz[3 * (size_t)v + a];
            p[c][a] = __fmul_rn(x, sc32);
            q[c][a] = __dmul_rn(double(x), sc);
            lo[a] = fminf(lo[a], fminf(p[c][a], __double2float_rd(q[c][a])));
            hi[a] = fmaxf(hi[a], fmaxf(p[c][a], __double2float_ru(q[c][a])));
        }
    }
    for (int a = 0; a < 3; ++a) {
        box[6 * slot + a] = lo[a];
        box[6 * slot + 3 + a] = hi[a];
    }
    float e1[3], e2[3];
    for (int a = 0; a < 3; ++a) {
        e1[a] = __fsub_rn(p[1][a], p[0][a]);
        e2[a] = __fsub_rn(p[2][a], p[0][a]);
    }
    const float nx = __fsub_rn(__fmul_rn(e1[1], e2[2]), __fmul_rn(e1[2], e2[1]));
    const float ny = -__fsub_rn(__fmul_rn(e1[0], e2[2]), __fmul_rn(e1[2], e2[0]));
    const float nz = __fsub_rn(__fmul_rn(e1[0], e2[1]), __fmul_rn(e1[1], e2[0]));
    const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(nx, nx), __fmul_rn(ny, ny)), __fmul_rn(nz, nz)));
    float n[3] = {0.0f, 0.0f, 0.0f};
    if (len > 0.0f) {
        n[0] = __fdiv_rn(nx, len);
        n[1] = __fdiv_rn(ny, len);
        n[2] = __fdiv_rn(nz, len);
    }
    GTri g;
    g.v0 = make_float4(p[0][0], p[0][1], p[0][2], n[0]);
    g.v1 = make_float4(p[1][0], p[1][1], p[1][2], n[1]);
    g.v2 = make_float4(p[2][0], p[2][1], p[2][2], n[2]);
    tris[slot] = g;
    if (tris64) {
        GTri64 h;
        for (int a = 0; a < 3; ++a) {
            h.v0[a] = q[0][a];
            h.e1[a] = __dsub_rn(q[1][a], q[0][a]);
            h.e2[a] = __dsub_rn(q[2][a], q[0][a]);
        }
        const double mx = __dsub_rn(__dmul_rn(h.e1[1], h.e2[2]), __dmul_rn(h.e1[2], h.e2[1]));
        const double my = -__dsub_rn(__dmul_rn(h.e1[0], h.e2[2]), __dmul_rn(h.e1[2], h.e2[0]));
        const double mz = __dsub_rn(__dmul_rn(h.e1[0], h.e2[1]), __dmul_rn(h.e1[1], h.e2[0]));
        const double l = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(mx, mx), __dmul_rn(my, my)), __dmul_rn(mz, mz)));
        if (l > 0.0) {
            h.n[0] = __ddiv_rn(mx, l);
            h.n[1] = __ddiv_rn(my, l);
            h.n[2] = __ddiv_rn(mz, l);
        } else {
            h.n[0] = h.n[1] = h.n[2] = 0.0;
        }
        tris64[slot] = h;
    }
}

__device__ __forceinline__ void grow(float (&lo)[3], float (&hi)[3], float lx, float ly, float lz, float hx, float hy,
                                     float hz) {
    lo[0] = fminf(lo[0], lx); lo[1] = fminf(lo[1], ly); lo[2] = fminf(lo[2], lz);
    hi[0] = fmaxf(hi[0], hx); hi[1] = fmaxf(hi[1], hy); hi[2] = fmaxf(hi[2], hz);
}

// Child references: >= 0 inner node, -1 empty slot (its far box is kept), other
// negative values leaves (~ref = first * 16 + count, count >= 1).
__global__ void k_refit_level(GNode4* nodes, const int32_t* __restrict__ level_nodes, int32_t n,
                              const float* __restrict__ box) {
    const int32_t i = blockIdx.x * (int32_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    GNode4* N = nodes + level_nodes[i];
    for (int c = 0; c < 4; ++c) {
        const int ref = (&N->child.x)[c];
        if (ref == -1) continue;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        if (ref < 0) {
            const int code = ~ref, first = code >> 4, cnt = code & 15;
            for (int k = 0; k < cnt; ++k) {
                const float* b = box + 6 * (int64_t)(first + k);
                grow(lo, hi, b[0], b[1], b[2], b[3], b[4], b[5]);
            }
        } else {
            const GNode4& C = nodes[ref];
            for (int cc = 0; cc < 4; ++cc) {
                if ((&C.child.x)[cc] == -1) continue;
                grow(lo, hi, (&C.lox.x)[cc], (&C.loy.x)[cc], (&C.loz.x)[cc], (&C.hix.x)[cc], (&C.hiy.x)[cc],
                     (&C.hiz.x)[cc]);
            }
        }
        (&N->lox.x)[c] = lo[0]; (&N->loy.x)[c] = lo[1]; (&N->loz.x)[c] = lo[2];
        (&N->hix.x)[c] = hi[0]; (&N->hiy.x)[c] = hi[1]; (&N->hiz.x)[c] = hi[2];
    }
}

}  // namespace
}  // namespace sbr

extern "C" sbr_status sbr_scene_update_vertices(sbr_scene* s, const float* xyz, size_t nverts) {
    using namespace sbr;
    if (!s || !xyz) return fail(SBR_ERR_INVALID_ARG, "scene and vertices are required");
    if (nverts * 3 != s->xyz.size()) return fail(SBR_ERR_INVALID_ARG, "vertex count differs from the scene's");
    for (size_t i = 0; i < 3 * nverts; ++i)
        if (!std::isfinite(xyz[i])) return fail(SBR_ERR_NONFINITE, "non-finite vertex coordinate");
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(s->device));
    sbr_status st = ensure_adjoint_data(s);  // device copies of the caller's vertices and triangles
    if (st != SBR_OK) return st;
    if (s->d_nodes8) {  // the opt-in 8-wide tree is not refitted: the sweep walks the 4-wide one again
        SBR_CUDA(cudaStreamSynchronize(s->stream));
        cudaFree(s->d_nodes8);
        s->d_nodes8 = nullptr;
        s->n_gnodes8 = 0;
    }
    if (!s->d_refit_nodes) {
        const size_t nb = s->refit_nodes.size() * sizeof(int32_t), bb = 6 * (size_t)s->ntris * sizeof(float);
        if (cudaMalloc(&s->d_refit_nodes, nb) != cudaSuccess || cudaMalloc(&s->d_tri_box, bb) != cudaSuccess)
            return fail(SBR_ERR_OOM, "refit buffers");
        SBR_CUDA(cudaMemcpy(s->d_refit_nodes, s->refit_nodes.data(), nb, cudaMemcpyHostToDevice));
        s->device_bytes += (int64_t)(nb + bb);
    }
    s->xyz.assign(xyz, xyz + 3 * nverts);
    cudaStream_t st_ = s->stream;
    SBR_CUDA(cudaMemcpyAsync(s->d_xyz, s->xyz.data(), s->xyz.size() * sizeof(float), cudaMemcpyHostToDevice, st_));
    const unsigned gt = (unsigned)((s->ntris + kRefitThreads - 1) / kRefitThreads);
    k_refit_tris<<<gt, kRefitThreads, 0, st_>>>(s->d_xyz, s->d_idx, s->d_tri_id, s->ntris, float(s->model_scale),
                                                 s->model_scale, s->d_tris, s->d_tris64, s->d_tri_box);
    SBR_CUDA(cudaGetLastError());
    const std::vector<int32_t>& off = s->refit_level_off;
    for (size_t d = off.size() - 1; d-- > 0;) {
        const int32_t n = off[d + 1] - off[d];
        if (n <= 0) continue;
        k_refit_level<<<(unsigned)((n + kRefitThreads - 1) / kRefitThreads), kRefitThreads, 0, st_>>>(
            s->d_nodes, s->d_refit_nodes + off[d], n, s->d_tri_box);
        SBR_CUDA(cudaGetLastError());
    }
    // the scene bounds (launcher clipping) from the root's slots
    GNode4 root;
    SBR_CUDA(cudaMemcpyAsync(&root, s->d_nodes, sizeof(GNode4), cudaMemcpyDeviceToHost, st_));
    SBR_CUDA(cudaStreamSynchronize(st_));
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < 4; ++c) {
        if ((&root.child.x)[c] == -1) continue;
        lo[0] = std::min(lo[0], double((&root.lox.x)[c])); hi[0] = std::max(hi[0], double((&root.hix.x)[c]));
        lo[1] = std::min(lo[1], double((&root.loy.x)[c])); hi[1] = std::max(hi[1], double((&root.hiy.x)[c]));
        lo[2] = std::min(lo[2], double((&root.loz.x)[c])); hi[2] = std::max(hi[2], double((&root.hiz.x)[c]));
    }
    for (int a = 0; a < 3; ++a) {
        s->aabb_lo[a] = lo[a];
        s->aabb_hi[a] = hi[a];
    }
    return SBR_OK;
}
