// gpu_build.cu -- binned SAH BVH build on the GPU, breadth first (one pass of
// kernels per tree level), producing the same tree as the host builder
// (bvh_build.cpp, the reference's algorithm family: src/scene/bvhBuilder.cpp:115-312).
//
// Why the trees match: every quantity that decides a split is order independent or
// computed with the host's operations in the host's order -- node and centroid
// bounds are exact minima / maxima, bin indices are int((c - c0) * (B / ext)) with
// each operation rounded alone, bin boxes are exact, and the SAH sweep runs on one
// thread in the host's axis / bin order with the same FP64 area and cost formulas.
// The partition is stable, so every node's triangle range stays sorted by triangle
// index (the ranges start as 0..N-1); the host's median fallback (all centroids
// equal: nth_element on (centroid, index)) is then the first half of the range.
// Only the order of triangles inside a leaf differs from the host build (which
// partitions with std::partition).
//
// Per level: big nodes (more than kWarpMax triangles) get their bounds and bins from
// grid-wide atomics (warp-aggregated), small nodes one warp each with bins in shared
// memory; then flags, one exclusive scan over all positions, a stable scatter, and
// child allocation.  Nodes are numbered breadth first on the device and renumbered
// in pre-order on the host.  One device-to-host read per level (the next level's
// node count); no kernel waits on another.
#include <algorithm>
#include <cfloat>
#include <vector>

#include "bvh_build.hpp"
#include "common.hpp"

namespace sbr {
namespace {

constexpr int kMaxBins = 32;
constexpr int kWarpMax = 512;   // nodes up to this many triangles are built by one warp
constexpr int kKeys = 7;        // per bin: lo x/y/z keys, hi x/y/z keys, count
constexpr int kScanBlock = 1024;

// Order-preserving map of floats to unsigned keys (min / max by integer atomics).
__device__ __forceinline__ unsigned fkey(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fval(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct Level {
    // active nodes of the level
    int32_t* node;          // global node id
    int32_t* s;             // triangle range [s, e)
    int32_t* e;
    unsigned* bounds;       // [12]: box lo keys, box hi keys, centroid lo keys, centroid hi keys
    int32_t* kind;          // 0 leaf, 1 SAH split, 2 median split
    int32_t* axis;
    int32_t* bin;
    int32_t* big_rank;      // -1: built by one warp
    int32_t* left_count;
    int32_t* child_slot;    // first of two slots in the next level
};

struct Work {
    const float* lo;        // [N * 3] triangle boxes
    const float* hi;
    const float* cen;       // [N * 3] centroids
    int32_t* idx;           // [N] position -> triangle
    int32_t* tmp;           // [N]
    int32_t* node_of;       // [N] position -> active slot (-1: in a finished leaf)
    int32_t* flag;          // [N]
    int32_t* scan;          // [N + 1]
    int32_t* block_sums;    // [N / kScanBlock + 2]
    unsigned* big_bins;     // [big nodes][3][B][kKeys]
    int32_t* counters;      // [0] big nodes, [1] next-level nodes, [2] node count
    // node records (breadth first ids)
    float* nlo;             // [2N * 3]
    float* nhi;
    int32_t* nleft;         // child ids, -1 for leaves
    int32_t* nright;
    int32_t* nfirst;
    int32_t* ncount;
    int n, bins, leaf_size, max_leaf;
};

__device__ __forceinline__ int bin_of(float c, float c0, float scl, int B) {
    const int b = __float2int_rz(__fmul_rn(__fsub_rn(c, c0), scl));
    return min(B - 1, max(0, b));
}

// Box area as the host computes it (Box::area, FP64, each operation rounded alone).
__device__ __forceinline__ double area_keys(const unsigned* lo, const unsigned* hi) {
    double d[3];
    for (int a = 0; a < 3; ++a) d[a] = fmax(0.0, __dsub_rn(double(fval(hi[a])), double(fval(lo[a]))));
    return __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[1]), __dmul_rn(d[1], d[2])), __dmul_rn(d[2], d[0])));
}

// The host builder's split decision (Builder::split) from filled bins [3][B][kKeys].
__device__ void sah_decide(const unsigned* bins, int B, const unsigned* bounds, int n, int leaf_size, int max_leaf,
                           int& kind, int& axis, int& bin) {
    kind = 0;
    axis = -1;
    bin = -1;
    if (n <= leaf_size) return;
    const double parent = area_keys(bounds, bounds + 3);
    double best = __longlong_as_double(0x7ff0000000000000LL);
    int bestAx = -1, bestBin = -1;
    for (int ax = 0; ax < 3; ++ax) {
        const float c0 = fval(bounds[6 + ax]), ext = __fsub_rn(fval(bounds[9 + ax]), c0);
        if (!(ext > 0.0f)) continue;
        const unsigned* bx = bins + ax * B * kKeys;
        // right-hand accumulations (b = B-1 .. 1), then the left sweep
        unsigned rlo[kMaxBins][3], rhi[kMaxBins][3];
        int rcnt[kMaxBins];
        unsigned alo[3] = {fkey(FLT_MAX), fkey(FLT_MAX), fkey(FLT_MAX)};
        unsigned ahi[3] = {fkey(-FLT_MAX), fkey(-FLT_MAX), fkey(-FLT_MAX)};
        int ac = 0;
        for (int b = B - 1; b > 0; --b) {
            for (int a = 0; a < 3; ++a) {
                alo[a] = min(alo[a], bx[b * kKeys + a]);
                ahi[a] = max(ahi[a], bx[b * kKeys + 3 + a]);
                rlo[b][a] = alo[a];
                rhi[b][a] = ahi[a];
            }
            ac += (int)bx[b * kKeys + 6];
            rcnt[b] = ac;
        }
        for (int a = 0; a < 3; ++a) { alo[a] = fkey(FLT_MAX); ahi[a] = fkey(-FLT_MAX); }
        ac = 0;
        for (int b = 0; b < B - 1; ++b) {
            for (int a = 0; a < 3; ++a) {
                alo[a] = min(alo[a], bx[b * kKeys + a]);
                ahi[a] = max(ahi[a], bx[b * kKeys + 3 + a]);
            }
            ac += (int)bx[b * kKeys + 6];
            if (ac == 0 || rcnt[b + 1] == 0) continue;
            const double cost = __ddiv_rn(__dadd_rn(__dmul_rn(area_keys(alo, ahi), double(ac)),
                                                    __dmul_rn(area_keys(rlo[b + 1], rhi[b + 1]), double(rcnt[b + 1]))),
                                          fmax(parent, 1e-300));
            if (cost < best) {
                best = cost;
                bestAx = ax;
                bestBin = b;
            }
        }
    }
    if (bestAx >= 0 && (best < double(n) || n > max_leaf)) {
        kind = 1;
        axis = bestAx;
        bin = bestBin;
    } else if (n > max_leaf) {
        kind = 2;  // all centroids equal: first half of the (index-sorted) range
    }
}

__device__ __forceinline__ void init_bins(unsigned* b, int count, int lane, int stride) {
    for (int i = lane; i < count; i += stride) {
        const int k = i % kKeys;
        b[i] = k < 3 ? fkey(FLT_MAX) : k < 6 ? fkey(-FLT_MAX) : 0u;
    }
}

__global__ void k_init(Work W, Level L) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < W.n) {
        W.idx[p] = p;
        W.node_of[p] = 0;
    }
    if (p == 0) {
        L.node[0] = 0;
        L.s[0] = 0;
        L.e[0] = W.n;
        W.counters[2] = 1;
    }
}

// Per active slot: reset bounds, pick big nodes and reset their bins.
__global__ void k_level_begin(Work W, Level L, int nact) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nact) return;
    for (int k = 0; k < 12; ++k) L.bounds[12 * j + k] = (k % 6) < 3 ? fkey(FLT_MAX) : fkey(-FLT_MAX);
    const int n = L.e[j] - L.s[j];
    L.big_rank[j] = n > kWarpMax ? atomicAdd(&W.counters[0], 1) : -1;
    if (L.big_rank[j] >= 0) init_bins(W.big_bins + (size_t)L.big_rank[j] * 3 * W.bins * kKeys, 3 * W.bins * kKeys, 0, 1);
}

// Big nodes: bounds by atomics, one warp-level reduction first when a whole warp
// works on one node (contiguous ranges make that the common case).
__global__ void k_big_bounds(Work W, Level L) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = p < W.n ? W.node_of[p] : -1;
    const bool mine = j >= 0 && L.big_rank[j] >= 0;
    const unsigned m = __ballot_sync(0xffffffffu, mine);
    if (!mine) return;
    unsigned v[12];
    const int t = W.idx[p];
    for (int a = 0; a < 3; ++a) {
        v[a] = fkey(W.lo[3 * t + a]);
        v[3 + a] = fkey(W.hi[3 * t + a]);
        v[6 + a] = fkey(W.cen[3 * t + a]);
        v[9 + a] = v[6 + a];
    }
    const int j0 = __shfl_sync(m, j, __ffs(m) - 1);
    const bool uniform = __all_sync(m, j == j0);
    unsigned* B = L.bounds + 12 * j;
    if (uniform) {
        for (int k = 0; k < 12; ++k)
            v[k] = (k % 6) < 3 ? __reduce_min_sync(m, v[k]) : __reduce_max_sync(m, v[k]);
        if ((threadIdx.x & 31) != __ffs(m) - 1) return;
    }
    for (int k = 0; k < 12; ++k) {
        if ((k % 6) < 3) atomicMin(B + k, v[k]);
        else atomicMax(B + k, v[k]);
    }
}

// Big nodes: bins on the three axes (shared-memory bins when the block's positions
// all belong to one node, else global atomics).
__global__ void k_big_bins(Work W, Level L) {
    extern __shared__ unsigned sb[];
    const int B = W.bins;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int p0 = blockIdx.x * blockDim.x, p1 = min(W.n, p0 + (int)blockDim.x) - 1;
    const int jf = W.node_of[p0], jl = W.node_of[p1];
    const bool block_uniform = jf >= 0 && jf == jl && L.big_rank[jf] >= 0;
    if (block_uniform) init_bins(sb, 3 * B * kKeys, threadIdx.x, blockDim.x);
    __syncthreads();
    const int j = p < W.n ? W.node_of[p] : -1;
    if (j >= 0 && L.big_rank[j] >= 0) {
        unsigned* bins = block_uniform ? sb : W.big_bins + (size_t)L.big_rank[j] * 3 * B * kKeys;
        const unsigned* bd = L.bounds + 12 * j;
        const int t = W.idx[p];
        for (int ax = 0; ax < 3; ++ax) {
            const float c0 = fval(bd[6 + ax]), ext = __fsub_rn(fval(bd[9 + ax]), c0);
            if (!(ext > 0.0f)) continue;
            const float scl = __fdiv_rn(float(B), ext);
            unsigned* bb = bins + (ax * B + bin_of(W.cen[3 * t + ax], c0, scl, B)) * kKeys;
            for (int a = 0; a < 3; ++a) {
                atomicMin(bb + a, fkey(W.lo[3 * t + a]));
                atomicMax(bb + 3 + a, fkey(W.hi[3 * t + a]));
            }
            atomicAdd(bb + 6, 1u);
        }
    }
    __syncthreads();
    if (block_uniform) {
        unsigned* g = W.big_bins + (size_t)L.big_rank[jf] * 3 * B * kKeys;
        for (int i = threadIdx.x; i < 3 * B * kKeys; i += blockDim.x) {
            const int k = i % kKeys;
            if (k < 3) atomicMin(g + i, sb[i]);
            else if (k < 6) atomicMax(g + i, sb[i]);
            else if (sb[i]) atomicAdd(g + i, sb[i]);
        }
    }
}

__global__ void k_big_split(Work W, Level L, int nact) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nact || L.big_rank[j] < 0) return;
    int kind, ax, bin;
    sah_decide(W.big_bins + (size_t)L.big_rank[j] * 3 * W.bins * kKeys, W.bins, L.bounds + 12 * j, L.e[j] - L.s[j],
               W.leaf_size, W.max_leaf, kind, ax, bin);
    L.kind[j] = kind;
    L.axis[j] = ax;
    L.bin[j] = bin;
}

// Small nodes: one warp each -- bounds, bins in shared memory, split decision.
__global__ void k_small(Work W, Level L, int nact) {
    extern __shared__ unsigned sb[];
    const int B = W.bins;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j = blockIdx.x * (blockDim.x >> 5) + warp;
    if (j >= nact || L.big_rank[j] >= 0) return;
    unsigned* bins = sb + warp * 3 * B * kKeys;
    const int s = L.s[j], e = L.e[j], n = e - s;
    unsigned v[12];
    for (int k = 0; k < 12; ++k) v[k] = (k % 6) < 3 ? fkey(FLT_MAX) : fkey(-FLT_MAX);
    for (int p = s + lane; p < e; p += 32) {
        const int t = W.idx[p];
        for (int a = 0; a < 3; ++a) {
            v[a] = min(v[a], fkey(W.lo[3 * t + a]));
            v[3 + a] = max(v[3 + a], fkey(W.hi[3 * t + a]));
            const unsigned c = fkey(W.cen[3 * t + a]);
            v[6 + a] = min(v[6 + a], c);
            v[9 + a] = max(v[9 + a], c);
        }
    }
    for (int k = 0; k < 12; ++k)
        v[k] = (k % 6) < 3 ? __reduce_min_sync(0xffffffffu, v[k]) : __reduce_max_sync(0xffffffffu, v[k]);
    if (lane < 12) L.bounds[12 * j + lane] = v[lane];
    if (n <= W.leaf_size) {
        if (lane == 0) L.kind[j] = 0;
        return;
    }
    init_bins(bins, 3 * B * kKeys, lane, 32);
    __syncwarp();
    for (int p = s + lane; p < e; p += 32) {
        const int t = W.idx[p];
        for (int ax = 0; ax < 3; ++ax) {
            const float c0 = fval(v[6 + ax]), ext = __fsub_rn(fval(v[9 + ax]), c0);
            if (!(ext > 0.0f)) continue;
            const float scl = __fdiv_rn(float(B), ext);
            unsigned* bb = bins + (ax * B + bin_of(W.cen[3 * t + ax], c0, scl, B)) * kKeys;
            for (int a = 0; a < 3; ++a) {
                atomicMin(bb + a, fkey(W.lo[3 * t + a]));
                atomicMax(bb + 3 + a, fkey(W.hi[3 * t + a]));
            }
            atomicAdd(bb + 6, 1u);
        }
    }
    __syncwarp();
    if (lane == 0) {
        int kind, ax, bin;
        sah_decide(bins, B, v, n, W.leaf_size, W.max_leaf, kind, ax, bin);
        L.kind[j] = kind;
        L.axis[j] = ax;
        L.bin[j] = bin;
    }
}

__global__ void k_flags(Work W, Level L) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= W.n) return;
    const int j = W.node_of[p];
    int f = 0;
    if (j >= 0) {
        const int kind = L.kind[j];
        if (kind == 1) {
            const int ax = L.axis[j];
            const unsigned* bd = L.bounds + 12 * j;
            const float c0 = fval(bd[6 + ax]), ext = __fsub_rn(fval(bd[9 + ax]), c0);
            const float scl = __fdiv_rn(float(W.bins), ext);
            f = bin_of(W.cen[3 * W.idx[p] + ax], c0, scl, W.bins) <= L.bin[j];
        } else if (kind == 2) {
            const int s = L.s[j], n = L.e[j] - s;
            f = (p - s) < n / 2;
        }
    }
    W.flag[p] = f;
}

// Exclusive scan of W.flag into W.scan[0..n] (three passes).
__global__ void k_scan_blocks(const int32_t* in, int32_t* out, int32_t* sums, int n) {
    __shared__ int32_t sh[kScanBlock];
    const int p = blockIdx.x * kScanBlock + threadIdx.x;
    const int x = p < n ? in[p] : 0;
    sh[threadIdx.x] = x;
    __syncthreads();
    for (int off = 1; off < kScanBlock; off <<= 1) {
        const int y = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
        __syncthreads();
        sh[threadIdx.x] += y;
        __syncthreads();
    }
    if (p < n) out[p] = sh[threadIdx.x] - x;
    if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = sh[threadIdx.x];
}
__global__ void k_scan_sums(int32_t* sums, int nb) {
    __shared__ int32_t carry;
    __shared__ int32_t sh[kScanBlock];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += kScanBlock) {
        const int i = base + threadIdx.x;
        const int x = i < nb ? sums[i] : 0;
        sh[threadIdx.x] = x;
        __syncthreads();
        for (int off = 1; off < kScanBlock; off <<= 1) {
            const int y = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
            __syncthreads();
            sh[threadIdx.x] += y;
            __syncthreads();
        }
        if (i < nb) sums[i] = carry + sh[threadIdx.x] - x;
        __syncthreads();
        if (threadIdx.x == kScanBlock - 1) carry += sh[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = carry;
}
__global__ void k_scan_add(int32_t* out, const int32_t* sums, int n, int nblk) {
    const int p = blockIdx.x * kScanBlock + threadIdx.x;
    if (p < n) out[p] += sums[blockIdx.x];
    if (p == n) out[n] = sums[nblk];  // the total
}

// Stable partition of every split node's range; other positions copy through.
__global__ void k_scatter(Work W, Level L) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= W.n) return;
    const int j = W.node_of[p];
    if (j < 0 || L.kind[j] == 0) {
        W.tmp[p] = W.idx[p];
        return;
    }
    const int s = L.s[j], e = L.e[j];
    const int base = W.scan[s];
    const int nl = W.scan[e] - base;
    const int lr = W.scan[p] - base;
    const int q = W.flag[p] ? s + lr : s + nl + (p - s - lr);
    W.tmp[q] = W.idx[p];
    if (p == s) L.left_count[j] = nl;
}

// Node records and the next level's active slots.
__global__ void k_emit(Work W, Level L, Level N, int nact, int cap) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nact) return;
    const int id = L.node[j];
    const unsigned* bd = L.bounds + 12 * j;
    for (int a = 0; a < 3; ++a) {
        W.nlo[3 * id + a] = fval(bd[a]);
        W.nhi[3 * id + a] = fval(bd[3 + a]);
    }
    const int s = L.s[j], e = L.e[j];
    if (L.kind[j] == 0) {
        W.nleft[id] = W.nright[id] = -1;
        W.nfirst[id] = s;
        W.ncount[id] = e - s;
        L.child_slot[j] = -1;
        return;
    }
    const int m = s + L.left_count[j];
    const int c = atomicAdd(&W.counters[1], 2);
    const int cid = atomicAdd(&W.counters[2], 2);
    if (c + 1 >= cap || cid + 1 >= 2 * W.n) {  // bounded by construction; never write past the arrays
        atomicOr(&W.counters[3], 1);
        L.child_slot[j] = -1;
        return;
    }
    W.nleft[id] = cid;
    W.nright[id] = cid + 1;
    W.nfirst[id] = 0;
    W.ncount[id] = 0;
    N.node[c] = cid;
    N.s[c] = s;
    N.e[c] = m;
    N.node[c + 1] = cid + 1;
    N.s[c + 1] = m;
    N.e[c + 1] = e;
    L.child_slot[j] = c;
}

__global__ void k_assign(Work W, Level L) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= W.n) return;
    const int j = W.node_of[p];
    if (j < 0) return;
    const int c = L.child_slot[j];
    W.node_of[p] = c < 0 ? -1 : (p < L.s[j] + L.left_count[j] ? c : c + 1);
}

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    return cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(count, 1));
}

}  // namespace

// See bvh_build.hpp.  Returns false (with the CUDA error in *err) if a CUDA call fails.
bool build_sah_gpu(const std::vector<float>& tri_lo, const std::vector<float>& tri_hi, const BuildOptions& opt,
                   cudaStream_t stream, BinTree& out, cudaError_t* err) {
    out = BinTree();
    const int n = (int)(tri_lo.size() / 3);
    if (n == 0) return true;
    const int B = std::min(std::max(2, opt.bin_count), kMaxBins);
    const int cap = std::min(n, 2 * (n / (opt.leaf_size + 1)) + 2);
    const int nblk = (n + kScanBlock - 1) / kScanBlock;
    std::vector<float> cen(3 * (size_t)n);
    for (size_t i = 0; i < 3 * (size_t)n; ++i) cen[i] = 0.5f * (tri_lo[i] + tri_hi[i]);

    Work W{};
    Level L[2]{};
    std::vector<void*> owned;
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** p, size_t count) {
        if (e == cudaSuccess) {
            e = dalloc(p, count);
            if (e == cudaSuccess) owned.push_back(*p);
        }
    };
    float *lo, *hi, *ce;
    A(&lo, 3 * (size_t)n);
    A(&hi, 3 * (size_t)n);
    A(&ce, 3 * (size_t)n);
    W.lo = lo;
    W.hi = hi;
    W.cen = ce;
    A(&W.idx, n);
    A(&W.tmp, n);
    A(&W.node_of, n);
    A(&W.flag, n);
    A(&W.scan, (size_t)n + 1);
    A(&W.block_sums, (size_t)nblk + 2);
    A(&W.big_bins, (size_t)(n / kWarpMax + 2) * 3 * B * kKeys);
    A(&W.counters, 4);
    A(&W.nlo, 3 * (size_t)(2 * n));
    A(&W.nhi, 3 * (size_t)(2 * n));
    A(&W.nleft, 2 * (size_t)n);
    A(&W.nright, 2 * (size_t)n);
    A(&W.nfirst, 2 * (size_t)n);
    A(&W.ncount, 2 * (size_t)n);
    for (Level& l : L) {
        A(&l.node, cap);
        A(&l.s, cap);
        A(&l.e, cap);
        A(&l.bounds, 12 * (size_t)cap);
        A(&l.kind, cap);
        A(&l.axis, cap);
        A(&l.bin, cap);
        A(&l.big_rank, cap);
        A(&l.left_count, cap);
        A(&l.child_slot, cap);
    }
    W.n = n;
    W.bins = B;
    W.leaf_size = opt.leaf_size;
    W.max_leaf = opt.max_leaf;
    auto cleanup = [&]() {
        for (void* p : owned) cudaFree(p);
    };
    if (e == cudaSuccess) e = cudaMemcpyAsync(lo, tri_lo.data(), 12 * (size_t)n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hi, tri_hi.data(), 12 * (size_t)n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ce, cen.data(), 12 * (size_t)n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(W.counters, 0, 4 * sizeof(int32_t), stream);
    if (e != cudaSuccess) {
        cleanup();
        *err = e;
        return false;
    }
    const int TB = 256;
    const int gp = (n + TB - 1) / TB;
    k_init<<<gp, TB, 0, stream>>>(W, L[0]);
    const size_t bin_bytes = (size_t)3 * B * kKeys * sizeof(unsigned);
    int nact = 1, cur = 0;
    while (nact > 0 && e == cudaSuccess) {
        Level& C = L[cur];
        Level& X = L[cur ^ 1];
        cudaMemsetAsync(W.counters, 0, 2 * sizeof(int32_t), stream);
        k_level_begin<<<(nact + TB - 1) / TB, TB, 0, stream>>>(W, C, nact);
        k_big_bounds<<<gp, TB, 0, stream>>>(W, C);
        k_big_bins<<<gp, TB, bin_bytes, stream>>>(W, C);
        k_big_split<<<(nact + TB - 1) / TB, TB, 0, stream>>>(W, C, nact);
        k_small<<<(nact + 7) / 8, 256, 8 * bin_bytes, stream>>>(W, C, nact);
        k_flags<<<gp, TB, 0, stream>>>(W, C);
        k_scan_blocks<<<nblk, kScanBlock, 0, stream>>>(W.flag, W.scan, W.block_sums, n);
        k_scan_sums<<<1, kScanBlock, 0, stream>>>(W.block_sums, nblk);
        k_scan_add<<<(n + 1 + kScanBlock - 1) / kScanBlock, kScanBlock, 0, stream>>>(W.scan, W.block_sums, n, nblk);
        k_scatter<<<gp, TB, 0, stream>>>(W, C);
        std::swap(W.idx, W.tmp);
        k_emit<<<(nact + TB - 1) / TB, TB, 0, stream>>>(W, C, X, nact, cap);
        k_assign<<<gp, TB, 0, stream>>>(W, C);
        int32_t cnt[4] = {0, 0, 0, 0};
        e = cudaMemcpyAsync(cnt, W.counters, sizeof(cnt), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess) e = cudaGetLastError();
        // cannot happen: each split node has more than leaf_size triangles
        if (e == cudaSuccess && (cnt[3] != 0 || cnt[1] > cap)) e = cudaErrorInvalidValue;
        const int next = cnt[1];
        nact = next;
        cur ^= 1;
    }
    int nnodes = 0;
    std::vector<int32_t> order(n);
    if (e == cudaSuccess) e = cudaMemcpy(&nnodes, W.counters + 2, sizeof(int32_t), cudaMemcpyDeviceToHost);
    std::vector<float> nlo, nhi;
    std::vector<int32_t> nl, nr, nf, nc;
    if (e == cudaSuccess) {
        nlo.resize(3 * (size_t)nnodes);
        nhi.resize(3 * (size_t)nnodes);
        nl.resize(nnodes);
        nr.resize(nnodes);
        nf.resize(nnodes);
        nc.resize(nnodes);
        e = cudaMemcpy(nlo.data(), W.nlo, 12 * (size_t)nnodes, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(nhi.data(), W.nhi, 12 * (size_t)nnodes, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(nl.data(), W.nleft, 4 * (size_t)nnodes, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(nr.data(), W.nright, 4 * (size_t)nnodes, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(nf.data(), W.nfirst, 4 * (size_t)nnodes, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(nc.data(), W.ncount, 4 * (size_t)nnodes, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(order.data(), W.idx, 4 * (size_t)n, cudaMemcpyDeviceToHost);
    }
    cleanup();
    if (e != cudaSuccess) {
        *err = e;
        return false;
    }
    // pre-order renumbering (left subtree before right), as the host builder's flatten
    out.nodes.reserve(nnodes);
    struct Item {
        int32_t id, parent, depth;
        bool right;
    };
    std::vector<Item> stack{{0, -1, 0, false}};
    while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        const int me = (int)out.nodes.size();
        BinNode b;
        for (int a = 0; a < 3; ++a) {
            b.lo[a] = nlo[3 * (size_t)it.id + a];
            b.hi[a] = nhi[3 * (size_t)it.id + a];
        }
        b.left = b.right = -1;
        b.first = nl[it.id] < 0 ? nf[it.id] : 0;
        b.count = nl[it.id] < 0 ? nc[it.id] : 0;
        out.nodes.push_back(b);
        out.depth = std::max(out.depth, it.depth + 1);
        if (it.parent >= 0) {
            if (it.right) out.nodes[it.parent].right = me;
            else out.nodes[it.parent].left = me;
        }
        if (nl[it.id] >= 0) {
            stack.push_back({nr[it.id], me, it.depth + 1, true});
            stack.push_back({nl[it.id], me, it.depth + 1, false});
        }
    }
    out.order = std::move(order);
    return true;
}

}  // namespace sbr
