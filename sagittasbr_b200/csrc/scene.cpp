// scene.cpp -- sbr_scene: mesh validation, BVH build, GPU layout and upload.
//
// Replaces the set-up half of runRcsApp (src/app/rtRcsEntry.cu:109-196):
// index checks, de-indexing with the model scale, buildBvh, and the device copies
// of triangles and nodes.  Errors are returned, never exit()-ed.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>

#include "bvh_build.hpp"
#include "plan.hpp"
#include "tie_order.hpp"

using namespace sbr;

namespace {

float round_down(double x) {
    float f = float(x);
    if (double(f) > x) f = std::nextafter(f, -INFINITY);
    return f;
}
float round_up(double x) {
    float f = float(x);
    if (double(f) < x) f = std::nextafter(f, INFINITY);
    return f;
}

// Triangle vertex in the reference FP32 build's arithmetic: float(position) * float(scale)
// (src/app/rtRcsEntry.cu:137-145 with Real = float).
inline void vert32(const float* xyz, uint32_t k, float sc, float out[3]) {
    for (int a = 0; a < 3; ++a) out[a] = xyz[3 * k + a] * sc;
}
// ... and in the FP64 build's: double(position) * double(scale).
inline void vert64(const float* xyz, uint32_t k, double sc, double out[3]) {
    for (int a = 0; a < 3; ++a) out[a] = double(xyz[3 * k + a]) * sc;
}

// fn(begin, end) over [0, n) in contiguous chunks on the host's threads (every
// element is written by exactly one thread, so the result does not depend on the
// thread count).
template <typename Fn>
void parallel_for(size_t n, int threads, Fn fn) {
    int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = (int)std::min<size_t>((size_t)nt, std::max<size_t>(1, n / 65536));
    if (nt <= 1) {
        fn(size_t(0), n);
        return;
    }
    std::vector<std::thread> pool;
    const size_t chunk = (n + nt - 1) / nt;
    for (int k = 0; k < nt; ++k) {
        const size_t b = k * chunk, e = std::min(n, b + chunk);
        if (b < e) pool.emplace_back(fn, b, e);
    }
    for (auto& t : pool) t.join();
}

void free_scene(sbr_scene* s) {
    if (!s) return;
    int cur = -1;
    cudaGetDevice(&cur);
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    cudaFree(s->d_nodes);
    cudaFree(s->d_nodes8);
    cudaFree(s->d_tris);
    cudaFree(s->d_tris64);
    cudaFree(s->d_tri_id);
    cudaFree(s->d_tie);
    cudaFree(s->d_xyz);
    cudaFree(s->d_idx);
    cudaFree(s->d_refit_nodes);
    cudaFree(s->d_tri_box);
    cudaFree(s->d_err);
    cudaFree(s->d_cancel);
    if (s->h_flag_vals) cudaFreeHost(s->h_flag_vals);
    if (s->cancel_stream) cudaStreamDestroy(s->cancel_stream);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (cur >= 0) cudaSetDevice(cur);
    delete s;
}

}  // namespace

namespace sbr {

sbr_status ensure_fp64(sbr_scene* s) {
    if (s->d_tris64) return SBR_OK;
    std::vector<GTri64> t64(s->ntris);
    for (int64_t slot = 0; slot < s->ntris; ++slot) {
        int32_t t = s->order[slot];
        double a[3], b[3], c[3];
        vert64(s->xyz.data(), s->idx[3 * t], s->model_scale, a);
        vert64(s->xyz.data(), s->idx[3 * t + 1], s->model_scale, b);
        vert64(s->xyz.data(), s->idx[3 * t + 2], s->model_scale, c);
        GTri64& g = t64[slot];
        for (int k = 0; k < 3; ++k) { g.v0[k] = a[k]; g.e1[k] = b[k] - a[k]; g.e2[k] = c[k] - a[k]; }
        double nx = g.e1[1] * g.e2[2] - g.e1[2] * g.e2[1];
        double ny = -(g.e1[0] * g.e2[2] - g.e1[2] * g.e2[0]);
        double nz = g.e1[0] * g.e2[1] - g.e1[1] * g.e2[0];
        double len = std::sqrt(nx * nx + ny * ny + nz * nz);
        if (len > 0) { g.n[0] = nx / len; g.n[1] = ny / len; g.n[2] = nz / len; }
        else { g.n[0] = g.n[1] = g.n[2] = 0.0; }
    }
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(s->device));
    size_t bytes = sizeof(GTri64) * t64.size();
    cudaError_t e = cudaMalloc(&s->d_tris64, bytes);
    if (e != cudaSuccess) return fail(SBR_ERR_OOM, "cudaMalloc of FP64 triangles failed");
    SBR_CUDA(cudaMemcpy(s->d_tris64, t64.data(), bytes, cudaMemcpyHostToDevice));
    s->device_bytes += (int64_t)bytes;
    return SBR_OK;
}

}  // namespace sbr

extern "C" {

sbr_status sbr_scene_create(const float* xyz, size_t nverts, const uint32_t* tri_idx, size_t ntris,
                            const sbr_build_opts* opts, sbr_scene** out) {
    if (!out) return fail(SBR_ERR_INVALID_ARG, "out is null");
    *out = nullptr;
    if (ntris == 0) return fail(SBR_ERR_EMPTY_MESH, "mesh contains no triangles");
    if (!xyz || !tri_idx || nverts == 0) return fail(SBR_ERR_INVALID_ARG, "null vertex or index array");
    if (ntris > (size_t(1) << 27)) return fail(SBR_ERR_TOO_LARGE, "more than 2^27 triangles");
    sbr_build_opts o{};
    if (opts) o = *opts;
    double scale = o.model_scale == 0.0 ? 1.0 : o.model_scale;
    if (!std::isfinite(scale)) return fail(SBR_ERR_NONFINITE, "model scale is not finite");
    if (o.node_width != 0 && o.node_width != 4 && o.node_width != 8)
        return fail(SBR_ERR_INVALID_ARG, "node_width must be 0, 4 or 8");
    for (size_t i = 0; i < 3 * ntris; ++i)
        if (tri_idx[i] >= nverts) return fail(SBR_ERR_BAD_INDEX, "triangle index out of range");
    for (size_t i = 0; i < 3 * nverts; ++i)
        if (!std::isfinite(xyz[i])) return fail(SBR_ERR_NONFINITE, "non-finite vertex coordinate");

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SBR_ERR_NO_DEVICE, "no CUDA device");
    int dev = o.device;
    if (dev < 0) SBR_CUDA(cudaGetDevice(&dev));
    if (dev >= ndev) return fail(SBR_ERR_INVALID_ARG, "device ordinal out of range");
    cudaDeviceProp prop;
    SBR_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) return fail(SBR_ERR_NO_DEVICE, "libsbr is built for sm_100a (B200); device is older");
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(dev));

    auto t0 = std::chrono::steady_clock::now();
    sbr_scene* s = new sbr_scene();
    s->device = dev;
    s->num_sms = prop.multiProcessorCount;
    s->ntris = (int64_t)ntris;
    s->model_scale = scale;
    s->xyz.assign(xyz, xyz + 3 * nverts);
    s->idx.assign(tri_idx, tri_idx + 3 * ntris);

    // per-triangle conservative boxes (cover both the FP32 and FP64 vertices)
    const float sc32 = float(scale);
    std::vector<float> lo(3 * ntris), hi(3 * ntris);
    parallel_for(ntris, o.n_threads, [&](size_t t0, size_t t1) {
        for (size_t t = t0; t < t1; ++t) {
            for (int a = 0; a < 3; ++a) { lo[3 * t + a] = INFINITY; hi[3 * t + a] = -INFINITY; }
            for (int c = 0; c < 3; ++c) {
                float p32[3];
                double p64[3];
                vert32(xyz, tri_idx[3 * t + c], sc32, p32);
                vert64(xyz, tri_idx[3 * t + c], scale, p64);
                for (int a = 0; a < 3; ++a) {
                    lo[3 * t + a] = std::min({lo[3 * t + a], p32[a], round_down(p64[a])});
                    hi[3 * t + a] = std::max({hi[3 * t + a], p32[a], round_up(p64[a])});
                }
            }
        }
    });
    BuildOptions bo;
    // 3, not the reference's 4 (src/scene/bvhBuilder.hpp:14): with 4-wide nodes one
    // more level of boxes is cheaper than a fourth triangle test per leaf (trihedral
    // +6 %, aircraft +4 %, SH ellipsoid +7 % on B200; 1 and 2 were no faster)
    bo.leaf_size = o.leaf_size > 0 ? std::min(o.leaf_size, kLeafMax) : 3;
    bo.bin_count = o.bin_count > 0 ? o.bin_count : 16;
    bo.n_threads = o.n_threads;
    bo.max_leaf = kLeafMax;
    const auto ts0 = std::chrono::steady_clock::now();
    BinTree tree;
    if (o.gpu_build > 0) {
        cudaStream_t bs = nullptr;
        cudaError_t be = cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking);
        const bool ok = be == cudaSuccess && build_sah_gpu(lo, hi, bo, bs, tree, &be);
        if (bs) cudaStreamDestroy(bs);
        if (!ok) {
            free_scene(s);
            return cuda_fail(be, "GPU BVH build");
        }
    } else {
        tree = build_sah(lo, hi, bo);
    }
    s->sah_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ts0).count();
    s->order = tree.order;
    s->n_bin_nodes = (int64_t)tree.nodes.size();
    s->depth = tree.depth;
    for (int a = 0; a < 3; ++a) { s->aabb_lo[a] = tree.nodes[0].lo[a]; s->aabb_hi[a] = tree.nodes[0].hi[a]; }

    // GPU nodes: the binary tree collapsed to 4-wide nodes.  A 4-wide node takes a
    // binary node's two children and keeps opening its largest (by surface area)
    // inner child until it holds four; siblings are stored contiguously, subtrees
    // depth first.
    std::vector<GNode4> g;
    std::vector<int32_t> level{0};  // depth of every 4-wide node (root 0), for refits
    auto leafRef = [](const BinNode& b) { return ~(b.first * 16 + b.count); };
    auto area = [](const BinNode& b) {
        float d0 = b.hi[0] - b.lo[0], d1 = b.hi[1] - b.lo[1], d2 = b.hi[2] - b.lo[2];
        return d0 * d1 + d1 * d2 + d2 * d0;
    };
    auto fill = [&](GNode4& n, int c, const BinNode* b, int ref) {
        const float far = 1e30f;
        float lo[3] = {far, far, far}, hi[3] = {far, far, far};
        if (b) for (int a = 0; a < 3; ++a) { lo[a] = b->lo[a]; hi[a] = b->hi[a]; }
        (&n.lox.x)[c] = lo[0]; (&n.hix.x)[c] = hi[0];
        (&n.loy.x)[c] = lo[1]; (&n.hiy.x)[c] = hi[1];
        (&n.loz.x)[c] = lo[2]; (&n.hiz.x)[c] = hi[2];
        (&n.child.x)[c] = ref;
    };
    if (tree.nodes[0].left < 0) {
        GNode4 n;
        fill(n, 0, &tree.nodes[0], leafRef(tree.nodes[0]));
        for (int c = 1; c < 4; ++c) fill(n, c, nullptr, ~0);
        g.push_back(n);
    } else {
        // A walker entering a node may hold, per ancestor, one stack entry for each
        // ancestor child it did not enter; `need` is that bound on arrival, and a node
        // only opens children while need + (children - 1) stays within the walker's
        // stack capacity.
        struct Work {
            int32_t bin, slot, need, depth;
        };
        g.reserve(tree.nodes.size() / 2 + 1);
        level.reserve(tree.nodes.size() / 2 + 1);
        g.emplace_back();
        std::vector<Work> work{{0, 0, 0, 0}};
        while (!work.empty()) {
            const Work w = work.back();
            const int32_t b = w.bin, slot = w.slot;
            work.pop_back();
            int32_t kids[4] = {tree.nodes[b].left, tree.nodes[b].right, -1, -1};
            int nk = 2;
            while (nk < 4 && w.need + nk <= kStackDepth) {
                int best = -1;
                float ba = -1.0f;
                for (int k = 0; k < nk; ++k) {
                    const BinNode& K = tree.nodes[kids[k]];
                    if (K.left >= 0 && area(K) > ba) { ba = area(K); best = k; }
                }
                if (best < 0) break;
                const BinNode& K = tree.nodes[kids[best]];
                for (int k = nk; k > best + 1; --k) kids[k] = kids[k - 1];
                kids[best] = K.left;
                kids[best + 1] = K.right;
                ++nk;
            }
            GNode4 n;
            Work inner[4];
            int ni = 0;
            const int32_t need = w.need + nk - 1;
            for (int c = 0; c < 4; ++c) {
                if (c >= nk) { fill(n, c, nullptr, ~0); continue; }
                const BinNode& K = tree.nodes[kids[c]];
                if (K.left >= 0) {
                    const int32_t idx = (int32_t)g.size() + ni;
                    inner[ni++] = {kids[c], idx, need, w.depth + 1};
                    fill(n, c, &K, idx);
                } else {
                    fill(n, c, &K, leafRef(K));
                }
            }
            g[slot] = n;
            g.resize(g.size() + ni);
            level.resize(g.size());
            for (int q = 0; q < ni; ++q) level[inner[q].slot] = inner[q].depth;
            for (int q = ni - 1; q >= 0; --q) work.push_back(inner[q]);
        }
    }
    s->n_gnodes = (int64_t)g.size();

    // Opt-in 8-wide tree over the same leaves: the same greedy collapse, opening
    // the largest inner child until a node holds eight children (or the walker's
    // stack bound is reached).
    std::vector<GNode8> g8;
    if (o.node_width == 8) {
        auto fill8 = [&](GNode8& n, int c, const BinNode* b, int ref) { fill(n.q[c >> 2], c & 3, b, ref); };
        if (tree.nodes[0].left < 0) {
            GNode8 n;
            fill8(n, 0, &tree.nodes[0], leafRef(tree.nodes[0]));
            for (int c = 1; c < 8; ++c) fill8(n, c, nullptr, ~0);
            g8.push_back(n);
        } else {
            struct Work8 {
                int32_t bin, slot, need;
            };
            g8.reserve(tree.nodes.size() / 4 + 1);
            g8.emplace_back();
            std::vector<Work8> work{{0, 0, 0}};
            while (!work.empty()) {
                const Work8 w = work.back();
                work.pop_back();
                int32_t kids[8] = {tree.nodes[w.bin].left, tree.nodes[w.bin].right, -1, -1, -1, -1, -1, -1};
                int nk = 2;
                while (nk < 8 && w.need + nk <= kStackDepth) {
                    int best = -1;
                    float ba = -1.0f;
                    for (int k = 0; k < nk; ++k) {
                        const BinNode& K = tree.nodes[kids[k]];
                        if (K.left >= 0 && area(K) > ba) { ba = area(K); best = k; }
                    }
                    if (best < 0) break;
                    const BinNode& K = tree.nodes[kids[best]];
                    for (int k = nk; k > best + 1; --k) kids[k] = kids[k - 1];
                    kids[best] = K.left;
                    kids[best + 1] = K.right;
                    ++nk;
                }
                GNode8 n;
                Work8 inner[8];
                int ni = 0;
                const int32_t need = w.need + nk - 1;
                for (int c = 0; c < 8; ++c) {
                    if (c >= nk) { fill8(n, c, nullptr, ~0); continue; }
                    const BinNode& K = tree.nodes[kids[c]];
                    if (K.left >= 0) {
                        const int32_t idx = (int32_t)g8.size() + ni;
                        inner[ni++] = {kids[c], idx, need};
                        fill8(n, c, &K, idx);
                    } else {
                        fill8(n, c, &K, leafRef(K));
                    }
                }
                g8[w.slot] = n;
                g8.resize(g8.size() + ni);
                for (int q = ni - 1; q >= 0; --q) work.push_back(inner[q]);
            }
        }
    }
    s->n_gnodes8 = (int64_t)g8.size();
    // nodes grouped by depth (a refit recomputes the boxes deepest level first)
    {
        const int32_t maxd = *std::max_element(level.begin(), level.end());
        s->refit_level_off.assign((size_t)maxd + 2, 0);
        for (int32_t d : level) ++s->refit_level_off[(size_t)d + 1];
        for (size_t d = 1; d < s->refit_level_off.size(); ++d) s->refit_level_off[d] += s->refit_level_off[d - 1];
        std::vector<int32_t> fillp(s->refit_level_off.begin(), s->refit_level_off.end() - 1);
        s->refit_nodes.resize(g.size());
        for (size_t k = 0; k < g.size(); ++k) s->refit_nodes[(size_t)fillp[(size_t)level[k]]++] = (int32_t)k;
    }

    // leaf-ordered triangles: v0, v1, v2 in FP32 and the unit normal unit(e1 x e2)
    // with e1, e2 in the reference's FP32 arithmetic (src/cuda/rtKernels.cu:13-14,42)
    std::vector<GTri> tr(ntris);
    std::vector<int32_t> ids(ntris);
    parallel_for(ntris, o.n_threads, [&](size_t s0, size_t s1) {
        for (size_t slot = s0; slot < s1; ++slot) {
            int32_t t = s->order[slot];
            ids[slot] = t;
            float a[3], b[3], c[3];
            vert32(xyz, tri_idx[3 * t], sc32, a);
            vert32(xyz, tri_idx[3 * t + 1], sc32, b);
            vert32(xyz, tri_idx[3 * t + 2], sc32, c);
            float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
            float e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
            float nx = e1[1] * e2[2] - e1[2] * e2[1];
            float ny = -(e1[0] * e2[2] - e1[2] * e2[0]);
            float nz = e1[0] * e2[1] - e1[1] * e2[0];
            float len = std::sqrt(nx * nx + ny * ny + nz * nz);
            float n[3] = {0.0f, 0.0f, 0.0f};
            if (len > 0.0f) { n[0] = nx / len; n[1] = ny / len; n[2] = nz / len; }
            tr[slot].v0 = make_float4(a[0], a[1], a[2], n[0]);
            tr[slot].v1 = make_float4(b[0], b[1], b[2], n[1]);
            tr[slot].v2 = make_float4(c[0], c[1], c[2], n[2]);
        }
    });
    // exact ties: where the mesh holds a triangle twice with opposite windings, each
    // slot's rank in the reference's walk order decides which of two equally near
    // triangles a ray keeps (the reference keeps the last it tests)
    std::vector<int32_t> tie;
    if (has_opposed_twins(xyz, tri_idx, ntris)) {
        const std::vector<int32_t> rank = reference_walk_rank(xyz, tri_idx, ntris, scale, o.n_threads);
        tie.resize(ntris);
        for (size_t slot = 0; slot < ntris; ++slot) tie[slot] = rank[(size_t)s->order[slot]];
    }
    auto t1 = std::chrono::steady_clock::now();
    s->build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();

    auto bail = [&](sbr_status st) {
        free_scene(s);
        return st;
    };
    cudaError_t e;
    size_t nb = sizeof(GNode4) * g.size(), tb = sizeof(GTri) * tr.size(), ib = sizeof(int32_t) * ids.size();
    if ((e = cudaMalloc(&s->d_nodes, nb)) != cudaSuccess || (e = cudaMalloc(&s->d_tris, tb)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_tri_id, ib)) != cudaSuccess || (e = cudaMalloc(&s->d_err, sizeof(uint32_t))) != cudaSuccess)
        return bail(fail(SBR_ERR_OOM, std::string("device allocation failed: ") + cudaGetErrorString(e)));
    if ((e = cudaMemcpy(s->d_nodes, g.data(), nb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(s->d_tris, tr.data(), tb, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(s->d_tri_id, ids.data(), ib, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = clear_device_word(s->d_err)) != cudaSuccess)
        return bail(cuda_fail(e, "scene upload"));
    // cancel flag: a device word (the kernels poll it from L2); the host sets it with an
    // asynchronous copy on a side stream, which runs while the sweep kernel is resident
    if ((e = cudaMalloc(&s->d_cancel, sizeof(int32_t))) != cudaSuccess ||
        (e = clear_device_word(s->d_cancel)) != cudaSuccess)
        return bail(cuda_fail(e, "cancel flag"));
    if ((e = cudaHostAlloc(&s->h_flag_vals, 2 * sizeof(int32_t), cudaHostAllocDefault)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaHostAlloc(cancel values)"));
    s->h_flag_vals[0] = 1;
    s->h_flag_vals[1] = 0;
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&s->cancel_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaStreamCreate"));
    s->device_bytes = (int64_t)(nb + tb + ib);
    if (!tie.empty()) {
        if ((e = cudaMalloc(&s->d_tie, ib)) != cudaSuccess)
            return bail(fail(SBR_ERR_OOM, std::string("device allocation failed: ") + cudaGetErrorString(e)));
        if ((e = cudaMemcpy(s->d_tie, tie.data(), ib, cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(cuda_fail(e, "tie rank upload"));
        s->device_bytes += (int64_t)ib;
    }
    if (!g8.empty()) {
        const size_t nb8 = sizeof(GNode8) * g8.size();
        if ((e = cudaMalloc(&s->d_nodes8, nb8)) != cudaSuccess)
            return bail(fail(SBR_ERR_OOM, std::string("device allocation failed: ") + cudaGetErrorString(e)));
        if ((e = cudaMemcpy(s->d_nodes8, g8.data(), nb8, cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(cuda_fail(e, "8-wide node upload"));
        s->device_bytes += (int64_t)nb8;
    }
    if (o.want_fp64 > 0) {
        sbr_status st = ensure_fp64(s);
        if (st != SBR_OK) return bail(st);
    }
    *out = s;
    return SBR_OK;
}

sbr_status sbr_scene_destroy(sbr_scene* scene) {
    if (!scene) return fail(SBR_ERR_INVALID_ARG, "scene is null");
    free_scene(scene);
    return SBR_OK;
}

sbr_status sbr_scene_info_get(const sbr_scene* s, sbr_scene_info* out) {
    if (!s || !out) return fail(SBR_ERR_INVALID_ARG, "null argument");
    out->n_triangles = s->ntris;
    out->n_nodes_bin = s->n_bin_nodes;
    out->n_nodes_gpu = s->n_gnodes;
    out->device_bytes = s->device_bytes;
    for (int a = 0; a < 3; ++a) { out->aabb_lo[a] = s->aabb_lo[a]; out->aabb_hi[a] = s->aabb_hi[a]; }
    out->build_ms = s->build_ms;
    out->device = s->device;
    out->bvh_depth = s->depth;
    out->sah_ms = s->sah_ms;
    return SBR_OK;
}

sbr_status sbr_scene_cancel(sbr_scene* s) {
    if (!s) return fail(SBR_ERR_INVALID_ARG, "scene is null");
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(s->device));
    SBR_CUDA(cudaMemcpyAsync(s->d_cancel, &s->h_flag_vals[0], sizeof(int32_t), cudaMemcpyHostToDevice,
                             s->cancel_stream));
    return SBR_OK;
}

sbr_status sbr_scene_reset_cancel(sbr_scene* s) {
    if (!s) return fail(SBR_ERR_INVALID_ARG, "scene is null");
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(s->device));
    SBR_CUDA(cudaMemcpyAsync(s->d_cancel, &s->h_flag_vals[1], sizeof(int32_t), cudaMemcpyHostToDevice,
                             s->cancel_stream));
    SBR_CUDA(cudaStreamSynchronize(s->cancel_stream));
    return SBR_OK;
}

}  // extern "C"
