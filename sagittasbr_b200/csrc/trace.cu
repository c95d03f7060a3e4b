// trace.cu -- sm_100a kernels of the SBR hot path and the plan that launches them.
//
// One work item = a strip of 16x16-ray tiles of one (job, angle) segment.  A CTA
// (256 threads, one ray per thread, warp = 8x4 ray block) takes items from a
// device queue (persistent mode) or one item per CTA (per-angle mode), traces the
// rays through every bounce (trace.cuh) and folds the PO exit-ray term of every
// frequency of the job into per-thread FP64 sums.  At the end of an item the CTA
// reduces them in a fixed order and adds the item total, quantised to a per-
// frequency fixed-point unit, to int64 accumulators with atomicAdd.  Integer
// addition is associative, so the field is bitwise reproducible whatever order
// the items finish in (the reference adds FP32 block sums with float atomics,
// src/cuda/poKernels.cu:118-120, whose order changes run to run).
//
// Replaces launchRaysMultiBounce + integratePoMultiBounce (src/cuda/rtKernels.cu:105-158,
// src/cuda/poKernels.cu:66-121) and the per-angle loop of runSweep
// (src/app/sweep.cu:332-441).
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "plan.hpp"
#include "trace.cuh"

namespace sbr {

struct TraceParams {
    SceneView S;
    const Segment* segs;
    const int64_t* seg_item_base;  // [n_segs + 1]
    int32_t n_segs;
    int32_t k_begin, k_count;      // frequency sub-range of every job (k_count 0 -> all)
    int32_t count_stats;
    const JobConst* jobs;
    const FreqConst* freqs;
    int64_t item_begin, item_end;  // items handled by this launch
    unsigned long long* queue;     // persistent queue head (null -> one item per CTA)
    unsigned long long* acc;       // [n_samples * 2] fixed-point field accumulators
    unsigned long long* acc_stats; // [n_segs * 4]
    uint32_t* err;
    const volatile int32_t* cancel;
    sbr_ray_record* records;       // debug records (REC instantiation only)
};

constexpr int kMaxK = 128;   // frequencies per job
constexpr int kRegK = 4;     // per-lane accumulation up to this many frequencies

struct RayOut {
    int count;
    int queries;
    float amp;     // 2 cos(theta) R^n, 0 when the ray adds nothing
    float dist32;  // FP32 path (reference FP32 arithmetic)
    double L;      // FP64 path
    float cosT, Rn;
    double cosD, RnD;  // FP64 copies (SBR_PREC_FP64)
};

// ------------------------------------------------------------- one ray (FP32/mixed)
template <int PREC, bool REC>
__device__ __forceinline__ RayOut trace_ray_f(const SceneView& S, const Segment& G, const JobConst& J, int i, int j,
                                              uint32_t& err, sbr_ray_record* rec) {
    F3 o;
    double L = 0.0;
    if (PREC == SBR_PREC_FP32) {
        float u = __fdiv_rn(float(i) + 0.5f, float(J.nx));
        float v = __fdiv_rn(float(j) + 0.5f, float(J.ny));
        o = f3(G.llcf[0] + u * G.uf[0] + v * G.vf[0], G.llcf[1] + u * G.uf[1] + v * G.vf[1],
               G.llcf[2] + u * G.uf[2] + v * G.vf[2]);
    } else {
        double u = (double(i) + 0.5) * J.inv_nx;
        double v = (double(j) + 0.5) * J.inv_ny;
        o = f3(float(G.llc[0] + u * G.u[0] + v * G.v[0]), float(G.llc[1] + u * G.u[1] + v * G.v[1]),
               float(G.llc[2] + u * G.u[2] + v * G.v[2]));
        L = G.shift;
    }
    F3 d = f3(G.rdf[0], G.rdf[1], G.rdf[2]);
    float dist32 = 0.0f;
    int count = 0, queries = 0;
    F3 nl = f3(0, 0, 0), dl = f3(0, 0, 0);
    for (int b = 0; b < J.max_bounces; ++b) {
        float tB = 1e20f;
        int slot = Walker<false>::closest(S, o, d, 1.0e-3f, tB, err);
        ++queries;
        if (slot < 0) break;
        const GTri* T = S.tris + slot;
        F3 n = f3(__ldg(&T->p.w), __ldg(&T->e1.w), __ldg(&T->e2.w));
        nl = n;
        dl = d;
        ++count;
        if (PREC == SBR_PREC_FP32) dist32 += tB;
        else L += double(tB);
        if (REC && count <= SBR_MAX_REC) rec->tri[count - 1] = __ldg(S.tri_id + slot);
        F3 p = o + tB * d;
        float dn = 2.0f * dot(d, n);
        d = unit(d - dn * n);
        o = p + 1.0e-4f * n;
    }
    RayOut r;
    r.count = count;
    r.queries = queries;
    r.dist32 = dist32;
    r.L = (PREC == SBR_PREC_FP32) ? double(dist32) : L;
    float Rn = 1.0f;
    for (int b = 0; b < count; ++b) Rn *= J.reflf;
    float c = dot(nl, f3(-dl.x, -dl.y, -dl.z));
    r.cosT = c;
    r.Rn = Rn;
    r.cosD = c;
    r.RnD = Rn;
    r.amp = (count > 0 && c > 0.0f) ? 2.0f * c * Rn : 0.0f;
    if (REC) {
        rec->count = count;
        rec->flags = 1;
        rec->dist = r.L;
        rec->normal[0] = nl.x; rec->normal[1] = nl.y; rec->normal[2] = nl.z;
        rec->lastdir[0] = dl.x; rec->lastdir[1] = dl.y; rec->lastdir[2] = dl.z;
    }
    return r;
}

// ------------------------------------------------------------- one ray (FP64)
template <bool REC>
__device__ __forceinline__ RayOut trace_ray_d(const SceneView& S, const Segment& G, const JobConst& J, int i, int j,
                                              uint32_t& err, sbr_ray_record* rec, double& ampD) {
    double u = (double(i) + 0.5) / double(J.nx);
    double v = (double(j) + 0.5) / double(J.ny);
    D3 o{G.llc[0] + u * G.u[0] + v * G.v[0], G.llc[1] + u * G.u[1] + v * G.v[1], G.llc[2] + u * G.u[2] + v * G.v[2]};
    D3 d{-G.dir[0], -G.dir[1], -G.dir[2]};
    double L = G.shift;
    int count = 0, queries = 0;
    D3 nl{0, 0, 0}, dl{0, 0, 0};
    for (int b = 0; b < J.max_bounces; ++b) {
        double tB = 1e20;
        int slot = Walker<true>::closest(S, o, d, 1.0e-3, tB, err);
        ++queries;
        if (slot < 0) break;
        const GTri64& T = S.tris64[slot];
        D3 n{T.n[0], T.n[1], T.n[2]};
        nl = n;
        dl = d;
        ++count;
        L += tB;
        if (REC && count <= SBR_MAX_REC) rec->tri[count - 1] = __ldg(S.tri_id + slot);
        D3 p = o + tB * d;
        double dn = 2.0 * dot(d, n);
        d = unit(d - dn * n);
        o = p + 1.0e-4 * n;
    }
    RayOut r;
    r.count = count;
    r.queries = queries;
    r.L = L;
    r.dist32 = float(L);
    double Rn = 1.0;
    for (int b = 0; b < count; ++b) Rn *= J.refl;
    double c = dot(nl, D3{-dl.x, -dl.y, -dl.z});
    r.cosT = float(c);
    r.Rn = float(Rn);
    r.cosD = c;
    r.RnD = Rn;
    ampD = (count > 0 && c > 0.0) ? 2.0 * c * Rn : 0.0;
    r.amp = float(ampD);
    if (REC) {
        rec->count = count;
        rec->flags = 1;
        rec->dist = L;
        rec->normal[0] = float(nl.x); rec->normal[1] = float(nl.y); rec->normal[2] = float(nl.z);
        rec->lastdir[0] = float(dl.x); rec->lastdir[1] = float(dl.y); rec->lastdir[2] = float(dl.z);
    }
    return r;
}

// PO term of one ray at one frequency, added to (re, im).
//  FP32: the reference FP32 arithmetic (phase fmodf in FP32).
//  MIXED: phase 2 k L reduced in FP64 by two-constant Cody-Waite, sin/cos of the
//         reduced FP32 angle, magnitude in FP64.
//  FP64: the reference USE_DOUBLE arithmetic.
__device__ __forceinline__ void po_term(int prec, const FreqConst& F, const RayOut& r, double ampD, double& re,
                                        double& im) {
    if (prec == SBR_PREC_FP32) {
        const float twoPi = 6.28318548202514648438f;
        float phase = (2.0f * F.kf) * r.dist32;
        phase = fmodf(phase, twoPi);
        float mag = (F.scalef * 2.0f) * r.cosT * r.Rn;
        float s, c;
        sincosf(phase, &s, &c);
        re += double(-mag * s);
        im += double(mag * c);
    } else if (prec == SBR_PREC_MIXED) {
        const double twoPiHi = 6.283185307179586232;      // nearest double to 2 pi
        const double twoPiLo = 2.4492935982947064e-16;     // 2 pi - twoPiHi
        const double invTwoPi = 0.15915494309189534561;
        double ph = 2.0 * F.k * r.L;
        double q = rint(ph * invTwoPi);
        double red = fma(-q, twoPiHi, ph);
        red = fma(-q, twoPiLo, red);
        float s, c;
        __sincosf(float(red), &s, &c);
        double mag = F.scale * double(r.amp);
        re -= mag * double(s);
        im += mag * double(c);
    } else {
        const double twoPi = 2.0 * 3.14159265358979323846;
        double phase = fmod((2.0 * F.k) * r.L, twoPi);
        double mag = (F.scale * 2.0) * r.cosD * r.RnD;
        double s, c;
        sincos(phase, &s, &c);
        re += -mag * s;
        im += mag * c;
    }
}

__device__ __forceinline__ int find_segment(const int64_t* base, int n, int64_t item) {
    int lo = 0, hi = n;  // base[lo] <= item < base[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(base + mid) <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void add_fixed(unsigned long long* acc, double v, double invQ) {
    long long q = __double2ll_rn(v * invQ);
    if (q != 0) atomicAdd(acc, (unsigned long long)q);
}

template <int PREC, bool TRANSPOSED, bool REC>
__global__ void __launch_bounds__(kCtaThreads) k_trace(const TraceParams P) {
    __shared__ long long s_item;
    __shared__ int s_seg;
    __shared__ double2 s_part[kCtaThreads / 32][kMaxK];
    __shared__ unsigned s_cnt[kCtaThreads / 32][4];

    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t err = 0;
    int iter = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            long long item;
            if (P.queue) item = P.item_begin + (long long)atomicAdd(P.queue, 1ull);
            else item = (iter == 0) ? P.item_begin + blockIdx.x : P.item_end;
            if (item < P.item_end && P.cancel && (iter & 15) == 0 && *P.cancel != 0) {
                atomicOr(P.err, DEV_ERR_CANCEL);
                item = P.item_end;
            }
            s_item = item;
            s_seg = item < P.item_end ? find_segment(P.seg_item_base, P.n_segs, item) : -1;
        }
        __syncthreads();
        const long long item = s_item;
        const int seg = s_seg;
        __syncthreads();
        if (item >= P.item_end) break;
        ++iter;

        const Segment& G = P.segs[seg];
        const JobConst J = P.jobs[G.job];
        const int kb = P.k_count > 0 ? P.k_begin : 0;
        const int K = P.k_count > 0 ? P.k_count : J.n_freqs;
        const FreqConst* F = P.freqs + J.freq_base + kb;

        double accRe[TRANSPOSED ? kMaxK / 32 : kRegK], accIm[TRANSPOSED ? kMaxK / 32 : kRegK];
#pragma unroll
        for (int c = 0; c < (TRANSPOSED ? kMaxK / 32 : kRegK); ++c) { accRe[c] = 0.0; accIm[c] = 0.0; }
        unsigned cRays = 0, cHit = 0, cBounce = 0, cQuery = 0;

        const long long local = item - G.item_base;
        const int t0 = int(local) * G.tiles_per_item;
        const int t1 = min(t0 + G.tiles_per_item, G.tiles);
        for (int t = t0; t < t1; ++t) {
            const int tx = t % G.tiles_x, ty = t / G.tiles_x;
            const int ri = tx * kTileW + (w & 1) * 8 + (lane & 7);
            const int rj = ty * kTileH + (w >> 1) * 4 + (lane >> 3);
            const bool valid = ri < G.ni && rj < G.nj;
            RayOut r;
            r.count = 0; r.queries = 0; r.amp = 0.0f; r.L = 0.0; r.dist32 = 0.0f; r.cosT = 0.0f; r.Rn = 1.0f;
            r.cosD = 0.0; r.RnD = 1.0;
            double ampD = 0.0;
            if (valid) {
                const int i = G.i0 + ri, j = G.j0 + rj;
                sbr_ray_record* rec = nullptr;
                if (REC) rec = P.records + ((size_t)G.angle * J.nx * J.ny + (size_t)j * J.nx + i);
                if (PREC == SBR_PREC_FP64) r = trace_ray_d<REC>(P.S, G, J, i, j, err, rec, ampD);
                else {
                    r = trace_ray_f<PREC, REC>(P.S, G, J, i, j, err, rec);
                    ampD = double(r.amp);
                }
                cRays += 1;
                cHit += r.count > 0;
                cBounce += r.count;
                cQuery += r.queries;
            }
            if (!TRANSPOSED) {
                if (r.amp != 0.0f) {
#pragma unroll
                    for (int k = 0; k < kRegK; ++k)
                        if (k < K) po_term(PREC, F[k], r, ampD, accRe[k], accIm[k]);
                }
            } else {
                // every lane owns frequencies lane, lane + 32, ...; rays are visited
                // in lane order so the per-frequency sum order is fixed
                unsigned m = __ballot_sync(0xffffffffu, r.amp != 0.0f);
                while (m) {
                    const int src = __ffs(m) - 1;
                    m &= m - 1;
                    RayOut q;
                    q.amp = __shfl_sync(0xffffffffu, r.amp, src);
                    q.L = __shfl_sync(0xffffffffu, r.L, src);
                    q.dist32 = __shfl_sync(0xffffffffu, r.dist32, src);
                    q.cosT = __shfl_sync(0xffffffffu, r.cosT, src);
                    q.Rn = __shfl_sync(0xffffffffu, r.Rn, src);
                    if (PREC == SBR_PREC_FP64) {
                        q.cosD = __shfl_sync(0xffffffffu, r.cosD, src);
                        q.RnD = __shfl_sync(0xffffffffu, r.RnD, src);
                    }
                    double qa = __shfl_sync(0xffffffffu, ampD, src);
#pragma unroll
                    for (int c = 0; c < kMaxK / 32; ++c) {
                        const int k = c * 32 + lane;
                        if (k < K) po_term(PREC, F[k], q, qa, accRe[c], accIm[c]);
                    }
                }
            }
        }

        // ---- fold the item: lanes -> warp -> CTA in a fixed order
        if (!TRANSPOSED) {
#pragma unroll
            for (int k = 0; k < kRegK; ++k) {
                if (k < K) {
                    double a = accRe[k], b = accIm[k];
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) {
                        a += __shfl_xor_sync(0xffffffffu, a, off);
                        b += __shfl_xor_sync(0xffffffffu, b, off);
                    }
                    if (lane == 0) s_part[w][k] = make_double2(a, b);
                }
            }
        } else {
#pragma unroll
            for (int c = 0; c < kMaxK / 32; ++c) {
                const int k = c * 32 + lane;
                if (k < K) s_part[w][k] = make_double2(accRe[c], accIm[c]);
            }
        }
        cRays = __reduce_add_sync(0xffffffffu, cRays);
        cHit = __reduce_add_sync(0xffffffffu, cHit);
        cBounce = __reduce_add_sync(0xffffffffu, cBounce);
        cQuery = __reduce_add_sync(0xffffffffu, cQuery);
        if (lane == 0) {
            s_cnt[w][0] = cRays; s_cnt[w][1] = cHit; s_cnt[w][2] = cBounce; s_cnt[w][3] = cQuery;
        }
        __syncthreads();
        if (threadIdx.x < K) {
            const int k = threadIdx.x;
            double a = 0.0, b = 0.0;
#pragma unroll
            for (int ww = 0; ww < kCtaThreads / 32; ++ww) { a += s_part[ww][k].x; b += s_part[ww][k].y; }
            const long long s = G.sample_base + kb + k;
            const double iq = F[k].inv_quantum;
            add_fixed(P.acc + 2 * s, a, iq);
            add_fixed(P.acc + 2 * s + 1, b, iq);
        }
        if (P.count_stats && threadIdx.x >= 128 && threadIdx.x < 132) {
            const int c = threadIdx.x - 128;
            unsigned long long tot = 0;
#pragma unroll
            for (int ww = 0; ww < kCtaThreads / 32; ++ww) tot += s_cnt[ww][c];
            if (tot) atomicAdd(P.acc_stats + 4 * (size_t)seg + c, tot);
        }
    }
    if (err) atomicOr(P.err, err);
}

// Converts the fixed-point accumulators to fields and clears them (and the
// queue) so the plan can run again without a memset.
__global__ void k_finalize(long long n_samples, const double* __restrict__ quantum, unsigned long long* acc,
                           double* field, long long n_stats, unsigned long long* acc_stats,
                           unsigned long long* out_stats, unsigned long long* queue) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < n_samples) {
        double q = quantum[t];
        long long re = (long long)acc[2 * t], im = (long long)acc[2 * t + 1];
        field[2 * t] = double(re) * q;
        field[2 * t + 1] = double(im) * q;
        acc[2 * t] = 0ull;
        acc[2 * t + 1] = 0ull;
    }
    if (t < n_stats) {
        out_stats[t] = acc_stats[t];
        acc_stats[t] = 0ull;
    }
    if (t == 0) *queue = 0ull;
}

__global__ void k_fill_records(sbr_ray_record* r, long long n) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n) return;
    sbr_ray_record z;
    z.count = 0;
    z.flags = 0;
    z.dist = 0.0;
    for (int a = 0; a < 3; ++a) { z.normal[a] = 0.0f; z.lastdir[a] = 0.0f; }
    for (int a = 0; a < SBR_MAX_REC; ++a) z.tri[a] = -1;
    r[t] = z;
}

// --------------------------------------------------------------------- host
namespace {

template <int PREC, bool TR, bool REC>
const void* kernel_ptr() {
    return reinterpret_cast<const void*>(&k_trace<PREC, TR, REC>);
}

const void* pick_kernel(int prec, bool transposed, bool rec) {
    switch (prec) {
        case SBR_PREC_MIXED:
            if (rec) return transposed ? kernel_ptr<SBR_PREC_MIXED, true, true>() : kernel_ptr<SBR_PREC_MIXED, false, true>();
            return transposed ? kernel_ptr<SBR_PREC_MIXED, true, false>() : kernel_ptr<SBR_PREC_MIXED, false, false>();
        case SBR_PREC_FP32:
            if (rec) return transposed ? kernel_ptr<SBR_PREC_FP32, true, true>() : kernel_ptr<SBR_PREC_FP32, false, true>();
            return transposed ? kernel_ptr<SBR_PREC_FP32, true, false>() : kernel_ptr<SBR_PREC_FP32, false, false>();
        default:
            if (rec) return transposed ? kernel_ptr<SBR_PREC_FP64, true, true>() : kernel_ptr<SBR_PREC_FP64, false, true>();
            return transposed ? kernel_ptr<SBR_PREC_FP64, true, false>() : kernel_ptr<SBR_PREC_FP64, false, false>();
    }
}

sbr_status launch_trace(const void* fn, int grid, cudaStream_t st, const TraceParams& p) {
    void* args[] = {const_cast<TraceParams*>(&p)};
    SBR_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(kCtaThreads), args, 0, st));
    return SBR_OK;
}

}  // namespace

sbr_status plan_launch(sbr_plan* pl, bool records, sbr_ray_record* d_records) {
    const bool transposed = pl->k_max > kRegK;
    const void* fn = pick_kernel(pl->prec, transposed, records);
    TraceParams p{};
    p.S = pl->scene_view;
    p.segs = pl->d_segs;
    p.seg_item_base = pl->d_seg_base;
    p.n_segs = (int32_t)pl->n_segs;
    p.jobs = pl->d_jobs;
    p.freqs = pl->d_freqs;
    p.acc = pl->d_acc;
    p.acc_stats = pl->d_acc_stats;
    p.err = pl->d_err;
    p.cancel = pl->d_cancel;
    p.records = d_records;
    cudaStream_t st = pl->stream;
    int launches = 0;
    if (pl->n_items > 0) {
        if (pl->mode == SBR_MODE_BATCHED || records) {
            if (pl->persistent_grid <= 0) {
                int occ = 0;
                SBR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kCtaThreads, 0));
                int per = pl->ctas_per_sm > 0 ? pl->ctas_per_sm : std::max(1, occ);
                pl->persistent_grid = std::max(1, per * pl->num_sms);
            }
            p.k_begin = 0;
            p.k_count = 0;
            p.count_stats = 1;
            p.item_begin = 0;
            p.item_end = pl->n_items;
            p.queue = pl->d_queue;
            int grid = (int)std::min<long long>(pl->persistent_grid, pl->n_items);
            sbr_status s = launch_trace(fn, grid, st, p);
            if (s != SBR_OK) return s;
            ++launches;
        } else {
            // the reference loop: one trace + PO launch per (angle, frequency)
            p.queue = nullptr;
            for (size_t g = 0; g < pl->segs.size(); ++g) {
                const Segment& G = pl->segs[g];
                long long n = pl->seg_base[g + 1] - pl->seg_base[g];
                if (n == 0) continue;
                const JobConst& J = pl->jobs[G.job];
                for (int k = 0; k < J.n_freqs; ++k) {
                    p.k_begin = k;
                    p.k_count = 1;
                    p.count_stats = k == 0;
                    p.item_begin = pl->seg_base[g];
                    p.item_end = pl->seg_base[g + 1];
                    sbr_status s = launch_trace(fn, (int)n, st, p);
                    if (s != SBR_OK) return s;
                    ++launches;
                }
            }
        }
    }
    long long nmax = std::max<long long>(pl->n_samples, (long long)pl->n_segs * 4);
    nmax = std::max<long long>(nmax, 1);
    int blocks = (int)((nmax + 255) / 256);
    k_finalize<<<blocks, 256, 0, st>>>(pl->n_samples, pl->d_quantum, pl->d_acc, pl->d_field,
                                       (long long)pl->n_segs * 4, pl->d_acc_stats, pl->d_stats, pl->d_queue);
    SBR_CUDA(cudaGetLastError());
    ++launches;
    pl->launches = launches;
    return SBR_OK;
}

sbr_status fill_records(sbr_ray_record* d, long long n, cudaStream_t st) {
    if (n <= 0) return SBR_OK;
    k_fill_records<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d, n);
    SBR_CUDA(cudaGetLastError());
    return SBR_OK;
}

int max_freqs_per_job() { return kMaxK; }

}  // namespace sbr

// =========================================================================
// Allocation-free sweep (sbr_run_noalloc).  No counterpart in the reference.
//
// For callers that may not allocate device memory while they run (a fixed
// device-memory budget owned by a pool, or other streams that must not be
// stalled by the synchronisation cudaMalloc / cudaFree perform).  The scratch a
// sweep needs beyond the caller's scene and output arrays lives in one file-scope
// device array of fixed size; host code reaches it only through the address
// cudaGetSymbolAddress returns for the current device.
// =========================================================================
#include <mutex>

namespace sbr {
namespace {

// Layout of the scratch array (device side) and of its host staging copy.
struct NoallocTables {
    Segment segs[SBR_NOALLOC_MAX_ANGLES];
    int64_t seg_base[SBR_NOALLOC_MAX_ANGLES + 1];
    JobConst job;
    FreqConst freqs[kMaxK];
    double quantum[SBR_NOALLOC_MAX_SAMPLES];
};
struct NoallocScratch {
    NoallocTables tables;
    unsigned long long acc[2 * SBR_NOALLOC_MAX_SAMPLES];
    unsigned long long acc_stats[4 * SBR_NOALLOC_MAX_ANGLES];
    unsigned long long queue;
};
static_assert(sizeof(NoallocScratch) <= SBR_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

// The scratch itself: every GPU that loads libsbr holds it until exit.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SBR_NOALLOC_SCRATCH_BYTES];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;                           // one call at a time per process
void* g_noalloc_addr[kNoallocMaxDevices] = {};     // device address of the array, per device
NoallocTables g_noalloc_host;                      // host staging (static: no heap use per call)

// Collects the sweep tables straight into the fixed-size staging copy.
struct NoallocSink : TableSink {
    int n_jobs = 0, n_freqs = 0, n_segs = 0, n_samples = 0;
    bool job(const JobConst& j) override {
        if (n_jobs++ > 0) return false;
        g_noalloc_host.job = j;
        return true;
    }
    bool freq(const FreqConst& f) override {
        if (n_freqs >= kMaxK) return false;
        g_noalloc_host.freqs[n_freqs++] = f;
        return true;
    }
    bool segment(const Segment& g, int64_t next_item, const double* q, int nf) override {
        if (n_segs >= SBR_NOALLOC_MAX_ANGLES || n_samples + nf > SBR_NOALLOC_MAX_SAMPLES) return false;
        g_noalloc_host.segs[n_segs] = g;
        g_noalloc_host.seg_base[n_segs + 1] = next_item;
        for (int f = 0; f < nf; ++f) g_noalloc_host.quantum[n_samples + f] = q[f];
        n_samples += nf;
        ++n_segs;
        return true;
    }
};

// Set-up, once per device and with that device current: the device address of
// the scratch array.  (Host code must never pass g_noalloc_scratch itself to a
// kernel: on the host that name denotes a host-side stand-in.)
sbr_status noalloc_address(int dev, NoallocScratch** out) {
    if (dev < 0 || dev >= kNoallocMaxDevices) return fail(SBR_ERR_UNSUPPORTED, "device ordinal too large");
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
        g_noalloc_addr[dev] = p;
    }
    *out = reinterpret_cast<NoallocScratch*>(g_noalloc_addr[dev]);
    return SBR_OK;
}

}  // namespace
}  // namespace sbr

extern "C" sbr_status sbr_run_noalloc(sbr_scene* s, const sbr_job* job, double* d_field, uint64_t* d_stats,
                                      const sbr_run_opts* opts) {
    using namespace sbr;
    if (!s || !job || !d_field) return fail(SBR_ERR_INVALID_ARG, "scene, job and d_field are required");
    sbr_run_opts o{};
    if (opts) o = *opts;
    if (o.mode != SBR_MODE_BATCHED) return fail(SBR_ERR_UNSUPPORTED, "the allocation-free sweep runs batched only");
    sbr_status st = validate_run(s, job, 1, o);
    if (st != SBR_OK) return st;
    if (job->n_angles > SBR_NOALLOC_MAX_ANGLES)
        return fail(SBR_ERR_TOO_LARGE, "allocation-free sweep: more than SBR_NOALLOC_MAX_ANGLES (1024) angles");
    if (job->n_angles * job->n_freqs > SBR_NOALLOC_MAX_SAMPLES)
        return fail(SBR_ERR_TOO_LARGE, "allocation-free sweep: more than SBR_NOALLOC_MAX_SAMPLES (4096) samples");
    if (o.precision == SBR_PREC_FP64 && !s->d_tris64)
        return fail(SBR_ERR_UNSUPPORTED, "allocation-free FP64 sweep needs a scene created with want_fp64 = 1");

    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    SBR_CUDA(cudaSetDevice(s->device));
    NoallocScratch* D = nullptr;
    st = noalloc_address(s->device, &D);
    if (st != SBR_OK) return st;

    NoallocSink sink;
    g_noalloc_host.seg_base[0] = 0;
    TableTotals tot;
    st = build_tables(s, job, 1, o, sink, tot);
    if (st != SBR_OK) return st;

    cudaStream_t stream = o.stream ? (cudaStream_t)o.stream : s->stream;
    const size_t nseg = (size_t)sink.n_segs, nsamp = (size_t)sink.n_samples;
    // tables in; accumulators, counters and queue head cleared (the array keeps the last call's contents)
    SBR_CUDA(cudaMemcpyAsync(D->tables.segs, g_noalloc_host.segs, nseg * sizeof(Segment), cudaMemcpyHostToDevice,
                             stream));
    SBR_CUDA(cudaMemcpyAsync(D->tables.seg_base, g_noalloc_host.seg_base, (nseg + 1) * sizeof(int64_t),
                             cudaMemcpyHostToDevice, stream));
    SBR_CUDA(cudaMemcpyAsync(&D->tables.job, &g_noalloc_host.job, sizeof(JobConst), cudaMemcpyHostToDevice, stream));
    SBR_CUDA(cudaMemcpyAsync(D->tables.freqs, g_noalloc_host.freqs, (size_t)sink.n_freqs * sizeof(FreqConst),
                             cudaMemcpyHostToDevice, stream));
    SBR_CUDA(cudaMemcpyAsync(D->tables.quantum, g_noalloc_host.quantum, nsamp * sizeof(double),
                             cudaMemcpyHostToDevice, stream));
    SBR_CUDA(cudaMemsetAsync(D->acc, 0, 2 * nsamp * sizeof(unsigned long long), stream));
    SBR_CUDA(cudaMemsetAsync(D->acc_stats, 0, 4 * nseg * sizeof(unsigned long long), stream));
    SBR_CUDA(cudaMemsetAsync(&D->queue, 0, sizeof(unsigned long long), stream));

    if (tot.n_items > 0) {
        const void* fn = pick_kernel(o.precision, tot.k_max > kRegK, false);
        int occ = 0;
        SBR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kCtaThreads, 0));
        int per = o.ctas_per_sm > 0 ? o.ctas_per_sm : std::max(1, occ);
        TraceParams p{};
        p.S = s->view();
        p.segs = D->tables.segs;
        p.seg_item_base = D->tables.seg_base;
        p.n_segs = (int32_t)nseg;
        p.k_begin = 0;
        p.k_count = 0;
        p.count_stats = 1;
        p.jobs = &D->tables.job;
        p.freqs = D->tables.freqs;
        p.item_begin = 0;
        p.item_end = tot.n_items;
        p.queue = &D->queue;
        p.acc = D->acc;
        p.acc_stats = D->acc_stats;
        p.err = s->d_err;
        p.cancel = s->d_cancel;
        p.records = nullptr;
        int grid = (int)std::min<long long>((long long)per * s->num_sms, tot.n_items);
        st = launch_trace(fn, grid, stream, p);
        if (st != SBR_OK) return st;
    }
    long long nmax = std::max<long long>(std::max<long long>((long long)nsamp, 4LL * (long long)nseg), 1);
    k_finalize<<<(unsigned)((nmax + 255) / 256), 256, 0, stream>>>(
        (long long)nsamp, D->tables.quantum, D->acc, d_field, d_stats ? 4LL * (long long)nseg : 0LL, D->acc_stats,
        reinterpret_cast<unsigned long long*>(d_stats), &D->queue);
    SBR_CUDA(cudaGetLastError());
    SBR_CUDA(cudaStreamSynchronize(stream));

    uint32_t e = 0;
    SBR_CUDA(cudaMemcpy(&e, s->d_err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) SBR_CUDA(cudaMemset(s->d_err, 0, sizeof(e)));
    if (e & DEV_ERR_CANCEL) return fail(SBR_ERR_CANCELLED, "run cancelled");
    if (e & DEV_ERR_BUDGET) return fail(SBR_ERR_TIMEOUT, "traversal iteration budget exceeded");
    if (e & DEV_ERR_STACK) return fail(SBR_ERR_STACK, "traversal stack overflow");
    return SBR_OK;
}
