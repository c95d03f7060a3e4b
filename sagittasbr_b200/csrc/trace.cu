// trace.cu -- sm_100a kernels of the SBR hot path and the plan that launches them.
//
// One work item = a run of 4x8-ray blocks of one (job, angle) segment, owned by
// one warp.  Warps take items from a device queue (persistent grid), trace one
// 4x8 block of parallel rays at a time through every bounce (trace.cuh), and fold
// the PO exit-ray term of every frequency of the job into per-lane FP64 sums.  At
// the end of an item the warp reduces them in a fixed order and adds the total, quantised to a per-frequency fixed-point unit,
// to int64 accumulators with atomicAdd.  Integer addition is associative, so the
// field is bitwise reproducible whatever order the items finish in (the reference
// adds FP32 block sums with float atomics, src/cuda/poKernels.cu:118-120, whose
// order changes run to run).
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
#include "ray.cuh"

namespace sbr {

struct TraceParams {
    SceneView S;
    const Segment* segs;
    const int64_t* seg_item_base;  // [n_segs + 1]
    int32_t n_segs;
    int32_t k_begin, k_count;      // frequency sub-range of every job (k_count 0 -> all)
    int32_t count_stats;
    int32_t n_rep;                 // accumulator replicas per sample
    const JobConst* jobs;
    const FreqConst* freqs;
    int64_t item_begin, item_end;  // items handled by this launch
    unsigned long long* queue;     // work-queue head of this launch
    const SegPol* segpol;          // [n_segs], SBR_POL_HHVV plans only
    const SceneView* scenes;       // multi-scene plans: scene of JobConst::scene
    unsigned long long* acc;       // [n_samples][n_pol][n_rep][2] fixed-point field accumulators
    unsigned long long* acc_stats; // [n_segs * 4]
    uint32_t* err;
    const volatile int32_t* cancel;
    sbr_ray_record* records;       // debug records (REC instantiation only)
    unsigned long long* zbuf;      // first-hit buffer of the launch's chunk, or null (walk the BVH)
    const uint32_t* tile_cnt;      // with zbuf: triangles per tile of the chunk (0: every ray misses)
};

constexpr int kMaxK = 128;   // accumulation channels (frequencies x polarisations) per job
constexpr int kRegK = 4;     // per-lane accumulation up to this many channels

// Accumulator layouts of the PO epilogue.  A job's channels are its frequencies
// (scalar plans) or its (frequency, polarisation) pairs, channel 2k + p (HHVV plans).
//   EPI_LANE1, EPI_LANE4: every lane sums the terms of its own rays for up to 1 / 4
//                         channels (registers sized to the plan's channel count)
//   EPI_T64, EPI_T128:    lanes own channels lane, lane + 32, ...; each finished ray
//                         is broadcast to the warp (up to 64 / 128 channels)
enum : int { EPI_LANE1 = 0, EPI_LANE4 = 1, EPI_T64 = 2, EPI_T128 = 3 };
template <int EPI>
struct Epi {
    static constexpr bool kTransposed = EPI >= EPI_T64;
    static constexpr int kAcc = EPI == EPI_LANE1 ? 1 : EPI == EPI_LANE4 ? 4 : EPI == EPI_T64 ? 2 : 4;
    static constexpr int kChannels = kTransposed ? 32 * kAcc : kAcc;
};
inline int pick_epi(int channels) {
    return channels <= 1 ? EPI_LANE1 : channels <= kRegK ? EPI_LANE4 : channels <= 64 ? EPI_T64 : EPI_T128;
}
// Resident CTAs (of 4 warps) per SM the kernels are register-budgeted for, by
// epilogue layout: the walk is latency-bound (node loads from L1/L2), so resident
// warps matter, but the wide layouts hold more state.  Measured on B200: per-lane
// layouts, trihedral (1 channel) 50,993 / 49,455 / 47,565 samples/s at 8 / 7 / 6
// CTAs (64 / 72 / 80 registers); lane-owned layouts, aircraft (64 channels)
// 13,180 / 13,499 / 12,948.  SBR_TRACE_CTAS_PER_SM (build flag) overrides both.
// SBR_TRACE_SPECULATIVE=1 (build flag): the mixed scalar sweep walks with the
// speculative closest-hit walk (trace.cuh) instead of the per-lane while-while one.
#ifndef SBR_TRACE_SPECULATIVE
#define SBR_TRACE_SPECULATIVE 0
#endif
#ifndef SBR_TRACE_CTAS_PER_SM
#define SBR_TRACE_CTAS_PER_SM 0
#endif
template <int EPI>
constexpr int min_ctas_per_sm() {
    return SBR_TRACE_CTAS_PER_SM > 0 ? SBR_TRACE_CTAS_PER_SM : (EPI >= EPI_T64 ? 7 : 8);
}

// Polarised exit terms of a finished ray (SBR_POL_HHVV): the HH and VV amplitudes
// and the physical exit path L + (plane - s.p_last), i.e. the path from the launch
// plane to the last hit point and back to the plane (the scalar term uses 2 L).
// The last hit point is the ray origin minus its 1e-4 nudge.  Rays the scalar
// gate drops (no hit, or cos(theta) <= 0) add nothing here either.
__device__ __forceinline__ void pol_finish_f(RayOut& o, const RayF& r, const PolF& e, const SegPol& P,
                                             const Segment& G) {
    o.pa[0] = 0.0;
    o.pa[1] = 0.0;
    o.Lp = 0.0;
    if (o.amp == 0.0f) return;
    const float twoRn = 2.0f * o.Rn;
    const F3 eh = f3(float(P.eh[0]), float(P.eh[1]), float(P.eh[2]));
    const F3 ev = f3(float(P.ev[0]), float(P.ev[1]), float(P.ev[2]));
    o.pa[0] = double(pol_amp(eh, r.nl, r.dl, e.h, twoRn));
    o.pa[1] = double(pol_amp(ev, r.nl, r.dl, e.v, twoRn));
    const F3 p = fma3(-1.0e-4f, r.nl, r.o);
    o.Lp = r.L + P.plane - dot(D3{G.dir[0], G.dir[1], G.dir[2]}, D3{double(p.x), double(p.y), double(p.z)});
    split_f32(0.5 * o.Lp, o.Lh, o.Ll);
}
__device__ __forceinline__ void pol_finish_d(RayOut& o, const RayD& r, const PolD& e, const SegPol& P,
                                             const Segment& G) {
    o.pa[0] = 0.0;
    o.pa[1] = 0.0;
    o.Lp = 0.0;
    if (o.amp == 0.0f) return;
    const double twoRn = 2.0 * o.RnD;
    o.pa[0] = pol_amp(D3{P.eh[0], P.eh[1], P.eh[2]}, r.nl, r.dl, e.h, twoRn);
    o.pa[1] = pol_amp(D3{P.ev[0], P.ev[1], P.ev[2]}, r.nl, r.dl, e.v, twoRn);
    const D3 p = r.o - 1.0e-4 * r.nl;
    o.Lp = r.L + P.plane - dot(D3{G.dir[0], G.dir[1], G.dir[2]}, p);
    split_f32(0.5 * o.Lp, o.Lh, o.Ll);
}

// Polarised PO term of one ray at one frequency: phase k Lp, magnitude
// k A / (4 pi) * amplitude, added as (-mag sin, mag cos) like the scalar term.
//  MIXED: k Lp = 2 pi (k / pi) (Lp / 2) reduced in turns from the FP32 pair
//         (Lh, Ll) = Lp / 2 (sincos_mixed), summed without the factor k A / (4 pi)
//         like the scalar MIXED term.
//  FP64:  fmod and sincos in FP64.
__device__ __forceinline__ void po_term_pol(int prec, const FreqConst& F, double Lp, float Lh, float Ll, double amp,
                                            double& re, double& im) {
    if (prec == SBR_PREC_MIXED) {
        float s, c;
        sincos_mixed(F, Lh, Ll, s, c);
        re -= amp * double(s);
        im += amp * double(c);
    } else {
        double s, c;
        sincos(fmod(F.k * Lp, 2.0 * 3.14159265358979323846), &s, &c);
        const double mag = F.scale * amp;
        re -= mag * s;
        im += mag * c;
    }
}

// Accumulator units per unit of a lane sum: MIXED sums leave out k A / (4 pi).
template <int PREC>
__device__ __forceinline__ double fold_factor(const FreqConst& F) {
    return PREC == SBR_PREC_MIXED ? F.scale * F.inv_quantum : F.inv_quantum;
}

__device__ __forceinline__ void add_fixed(unsigned long long* acc, double v, double invQ) {
    const long long q = __double2ll_rn(v * invQ);
    if (q != 0) atomicAdd(acc, (unsigned long long)q);
}

// Warp-persistent sweep kernel.  Every warp independently takes a work item (a
// run of 4x8-ray blocks of one (job, angle) segment) and traces it one block at a
// time, all lanes at the same bounce (no CTA-wide barrier anywhere).  Each lane
// folds the PO terms of its finished rays into FP64 sums (MIXED lane-owned
// layouts: through FP32 partial sums of one 4x8 block); at the end of the item
// the warp reduces them in a fixed order and adds the total, as int64 fixed
// point, to one of the segment's accumulator replicas.  Which lane takes which
// ray depends only on the item, so every sum is reproducible bit for bit.
template <int PREC, int EPI, bool REC, bool POL, bool MULTI, bool W8 = false>
__global__ void __launch_bounds__(kCtaThreads, min_ctas_per_sm<EPI>()) k_trace(const TraceParams P) {
    constexpr unsigned FULL = 0xffffffffu;
    constexpr bool F64 = PREC == SBR_PREC_FP64;
    constexpr bool TRANSPOSED = Epi<EPI>::kTransposed;
    constexpr int NACC = Epi<EPI>::kAcc;
    constexpr int NPOL = POL ? 2 : 1;
    const int lane = threadIdx.x & 31;
    const int warp_global = (int)((blockIdx.x * (unsigned)kCtaThreads + threadIdx.x) >> 5);
    // MIXED lane-owned epilogues sum each block's terms (at most 32 per channel) in
    // FP32 and add the block partials to the FP64 sums: the FP32 pair phase, one
    // sine / cosine and two FMAs per (ray, channel), no conversions.  Their FP64
    // sums stay in registers (measured on B200 against shared memory: aircraft
    // 14,198 vs 14,035 samples/s, HH + VV aircraft 11,689 vs 11,268).  The FP32 /
    // FP64 polarised lane-owned epilogues, which add every term to the FP64 sums,
    // keep those in shared memory (lane-owned, no atomics), leaving registers to the
    // walk and the E vectors.
    constexpr bool PART = TRANSPOSED && PREC == SBR_PREC_MIXED;
    constexpr bool SACC = TRANSPOSED && POL && !PART;
    __shared__ double2 s_acc[SACC ? (kCtaThreads / 32) * NACC * 32 : 1];
    double2* const my_acc = s_acc + (SACC ? (threadIdx.x >> 5) * NACC * 32 + lane : 0);
    const int rep = warp_global % P.n_rep;
    uint32_t err = 0;
    int iter = 0;
    for (;;) {
        long long item = 0;
        if (lane == 0) {
            item = P.item_begin + (long long)atomicAdd(P.queue, 1ull);
            if (item < P.item_end && P.cancel && (iter & 15) == 0 && *P.cancel != 0) {
                atomicOr(P.err, DEV_ERR_CANCEL);
                item = P.item_end;
            }
        }
        item = __shfl_sync(FULL, item, 0);
        if (item >= P.item_end) break;
        ++iter;

        const int seg = find_segment(P.seg_item_base, P.n_segs, item);
        const Segment& G = P.segs[seg];
        const JobConst J = P.jobs[G.job];
        const SceneView S = MULTI ? P.scenes[J.scene] : P.S;
        const int kb = P.k_count > 0 ? P.k_begin : 0;
        const int K = P.k_count > 0 ? P.k_count : J.n_freqs;
        const FreqConst* F = P.freqs + J.freq_base + kb;
        const int b0 = int(item - G.item_base) * G.blocks_per_item;
        const int nslots = min(G.blocks_per_item, G.blocks - b0) * 32;
        const int i_end = G.i0 + G.ni, j_end = G.j0 + G.nj;
        const int KC = K * NPOL;  // channels of this item

        double accRe[SACC ? 1 : NACC], accIm[SACC ? 1 : NACC];
        float pRe[PART ? NACC : 1], pIm[PART ? NACC : 1];
#pragma unroll
        for (int c = 0; c < NACC; ++c) {
            if constexpr (SACC) my_acc[c * 32] = make_double2(0.0, 0.0);
            else { accRe[c] = 0.0; accIm[c] = 0.0; }
            if constexpr (PART) { pRe[c] = 0.0f; pIm[c] = 0.0f; }
        }
        unsigned cRays = 0, cHit = 0, cBounce = 0, cQuery = 0;

        RayF rf;
        RayD rd;
        PolF ef;
        PolD ed;
        const SegPol* GP = POL ? P.segpol + seg : nullptr;
        bool active = false;
        int queries = 0;
        sbr_ray_record* rec = nullptr;
        int next = 0;  // next slot of the item to hand out (same value in every lane)

        auto refill = [&]() {
            for (;;) {
                const unsigned need = __ballot_sync(FULL, !active);
                if (need == 0 || next >= nslots) break;
                if (!REC && P.tile_cnt != nullptr && need == FULL) {
                    // full blocks whose tile no triangle reaches: all 32 rays miss their
                    // first query (counted as launched and queried, nothing else to do).
                    // Only blocks inside the grid are skipped: the lanes a ragged block
                    // leaves idle take the next block's first slots, and skipping it would
                    // regroup the rays that follow into other FP32 partial sums.  So
                    // `next` stays block-aligned here.
                    while (next < nslots && (next & 31) == 0) {
                        const int blk = b0 + (next >> 5);
                        const int bi = (blk % G.blocks_x) * kBlockW, bj = (blk / G.blocks_x) * kBlockH;
                        if (bi + kBlockW > G.ni || bj + kBlockH > G.nj || P.tile_cnt[G.tbase + blk] != 0u) break;
                        ++cRays;
                        ++cQuery;
                        next += 32;
                    }
                    if (next >= nslots) break;
                }
                const int s = next + __popc(need & ((1u << lane) - 1u));
                if (!active && s < nslots) {
                    const int blk = b0 + (s >> 5), l = s & 31;
                    const int i = G.i0 + (blk % G.blocks_x) * kBlockW + (l % kBlockW);
                    const int j = G.j0 + (blk / G.blocks_x) * kBlockH + (l / kBlockW);
                    if (i < i_end && j < j_end) {
                        if (F64) start_d(rd, G, J, i, j);
                        else start_f<PREC>(rf, G, J, i, j);
                        if constexpr (POL) {
                            if (F64) {
                                ed.h = D3{GP->eh[0], GP->eh[1], GP->eh[2]};
                                ed.v = D3{GP->ev[0], GP->ev[1], GP->ev[2]};
                            } else {
                                ef.h = f3(float(GP->eh[0]), float(GP->eh[1]), float(GP->eh[2]));
                                ef.v = f3(float(GP->ev[0]), float(GP->ev[1]), float(GP->ev[2]));
                            }
                        }
                        active = true;
                        queries = 0;
                        ++cRays;
                        if (REC) rec = P.records + ((size_t)G.angle * J.nx * J.ny + (size_t)j * J.nx + i);
                    }
                }
                next += __popc(need);
            }
        };

        refill();
        while (__any_sync(FULL, active)) {
            bool done = false;
            RayOut out;
            out.amp = 0.0f;
            // the speculative walk is entered by the active lanes together (first hits
            // from the raster buffer skip the walk, so it is not used with one)
            constexpr bool SPEC = SBR_TRACE_SPECULATIVE && PREC == SBR_PREC_MIXED && !REC && !POL && !W8;
            const unsigned amask = SPEC ? __ballot_sync(FULL, active) : 0u;
            if (active) {
                if constexpr (SPEC) {
                    done = P.zbuf == nullptr
                               ? step_f<PREC, REC, POL, W8, true>(rf, ef, S, J.max_bounces, err, rec, nullptr, amask)
                               : step_f<PREC, REC, POL, W8>(rf, ef, S, J.max_bounces, err, rec, P.zbuf);
                } else {
                    done = F64 ? step_d<REC, POL>(rd, ed, S, J.max_bounces, err, rec)
                               : step_f<PREC, REC, POL, W8>(rf, ef, S, J.max_bounces, err, rec, P.zbuf);
                }
                ++queries;
                if (done) {
                    const int cnt = F64 ? rd.count : rf.count;
                    out = F64 ? finish_d(rd, J) : finish_f<PREC>(rf, J);
                    if constexpr (POL) {
                        if (F64) pol_finish_d(out, rd, ed, *GP, G);
                        else pol_finish_f(out, rf, ef, *GP, G);
                    }
                    cHit += cnt > 0;
                    cBounce += cnt;
                    cQuery += queries;
                    active = false;
                    if (REC) {
                        rec->count = cnt;
                        rec->flags = 1;
                        rec->dist = out.L;
                        if (F64) {
                            rec->normal[0] = float(rd.nl.x); rec->normal[1] = float(rd.nl.y); rec->normal[2] = float(rd.nl.z);
                            rec->lastdir[0] = float(rd.dl.x); rec->lastdir[1] = float(rd.dl.y); rec->lastdir[2] = float(rd.dl.z);
                        } else {
                            rec->normal[0] = rf.nl.x; rec->normal[1] = rf.nl.y; rec->normal[2] = rf.nl.z;
                            rec->lastdir[0] = rf.dl.x; rec->lastdir[1] = rf.dl.y; rec->lastdir[2] = rf.dl.z;
                        }
                    }
                }
            }
            if constexpr (!TRANSPOSED) {
                if (done && out.amp != 0.0f) {
#pragma unroll
                    for (int ch = 0; ch < NACC; ++ch) {
                        if (ch < KC) {
                            if constexpr (POL)
                                po_term_pol(PREC, F[ch >> 1], out.Lp, out.Lh, out.Ll, out.pa[ch & 1], accRe[ch], accIm[ch]);
                            else po_term(PREC, F[ch], out, accRe[ch], accIm[ch]);
                        }
                    }
                }
            } else if constexpr (PART) {
                // lanes own channels lane, lane + 32, ...; finished rays are taken
                // in lane order, so every channel's sum has a fixed order.  Per
                // (ray, channel): the phase in FP32 pairs, one sine and cosine, two
                // FP32 FMAs into the block's partial sums
                unsigned m = __ballot_sync(FULL, done && out.amp != 0.0f);
                const float a0 = POL ? float(out.pa[0]) : out.amp;
                const float a1 = POL ? float(out.pa[1]) : 0.0f;
                while (m) {
                    const int src = __ffs(m) - 1;
                    m &= m - 1;
                    const float qa0 = __shfl_sync(FULL, a0, src);
                    const float qa1 = POL ? __shfl_sync(FULL, a1, src) : 0.0f;
                    const float Lh = __shfl_sync(FULL, out.Lh, src), Ll = __shfl_sync(FULL, out.Ll, src);
                    const float a = (POL && (lane & 1)) ? qa1 : qa0;  // channel 2k + p takes polarisation p
#pragma unroll
                    for (int c = 0; c < NACC; ++c) {
                        const int ch = c * 32 + lane;
                        if (ch < KC) {
                            float sn, cs;
                            sincos_mixed(F[POL ? ch >> 1 : ch], Lh, Ll, sn, cs);
                            pRe[c] = fmaf(-a, sn, pRe[c]);
                            pIm[c] = fmaf(a, cs, pIm[c]);
                        }
                    }
                }
            } else {
                // the same broadcast with the FP32 / FP64 terms summed in FP64
                unsigned m = __ballot_sync(FULL, done && out.amp != 0.0f);
                while (m) {
                    const int src = __ffs(m) - 1;
                    m &= m - 1;
                    RayOut q;
                    if constexpr (POL) {
                        q.pa[0] = __shfl_sync(FULL, out.pa[0], src);
                        q.pa[1] = __shfl_sync(FULL, out.pa[1], src);
                        q.Lp = __shfl_sync(FULL, out.Lp, src);
                    } else {
                        q.amp = __shfl_sync(FULL, out.amp, src);
                        q.L = __shfl_sync(FULL, out.L, src);
                        q.dist32 = __shfl_sync(FULL, out.dist32, src);
                        q.cosT = __shfl_sync(FULL, out.cosT, src);
                        q.Rn = __shfl_sync(FULL, out.Rn, src);
                        q.cosD = F64 ? __shfl_sync(FULL, out.cosD, src) : 0.0;
                        q.RnD = F64 ? __shfl_sync(FULL, out.RnD, src) : 0.0;
                    }
#pragma unroll
                    for (int c = 0; c < NACC; ++c) {
                        const int ch = c * 32 + lane;
                        if (ch < KC) {
                            if constexpr (SACC)
                                po_term_pol(PREC, F[ch >> 1], q.Lp, 0.0f, 0.0f, q.pa[ch & 1], my_acc[c * 32].x,
                                            my_acc[c * 32].y);
                            else if constexpr (POL)
                                po_term_pol(PREC, F[ch >> 1], q.Lp, 0.0f, 0.0f, q.pa[ch & 1], accRe[c], accIm[c]);
                            else po_term(PREC, F[ch], q, accRe[c], accIm[c]);
                        }
                    }
                }
            }
            // the next 4x8 block starts when the whole warp is done with this one:
            // keeping the warp's rays at the same bounce keeps them coherent (they
            // share direction and walk the same nodes), which is worth more than
            // refilling idle lanes
            if (!__any_sync(FULL, active)) {
                if constexpr (PART) {
#pragma unroll
                    for (int c = 0; c < NACC; ++c) {
                        if constexpr (SACC) {
                            my_acc[c * 32].x += double(pRe[c]);
                            my_acc[c * 32].y += double(pIm[c]);
                        } else {
                            accRe[c] += double(pRe[c]);
                            accIm[c] += double(pIm[c]);
                        }
                        pRe[c] = 0.0f;
                        pIm[c] = 0.0f;
                    }
                }
                refill();
            }
        }

        // ---- fold the item: lanes -> warp in a fixed order, then fixed point.
        // Channel ch of sample (sbase + k) lives at accumulator (sbase * NPOL + ch).
        const long long cbase = (G.sample_base + kb) * NPOL;
        if constexpr (!TRANSPOSED) {
#pragma unroll
            for (int ch = 0; ch < NACC; ++ch) {
                if (ch < KC) {
                    double a = accRe[ch], b = accIm[ch];
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) {
                        a += __shfl_xor_sync(FULL, a, off);
                        b += __shfl_xor_sync(FULL, b, off);
                    }
                    if (lane == ch) {
                        const double invQ = fold_factor<PREC>(F[POL ? ch >> 1 : ch]);
                        unsigned long long* A = P.acc + 2 * ((cbase + ch) * P.n_rep + rep);
                        add_fixed(A, a, invQ);
                        add_fixed(A + 1, b, invQ);
                    }
                }
            }
        } else {
#pragma unroll
            for (int c = 0; c < NACC; ++c) {
                const int ch = c * 32 + lane;
                if (ch < KC) {
                    const double invQ = fold_factor<PREC>(F[POL ? ch >> 1 : ch]);
                    unsigned long long* A = P.acc + 2 * ((cbase + ch) * P.n_rep + rep);
                    if constexpr (SACC) {
                        add_fixed(A, my_acc[c * 32].x, invQ);
                        add_fixed(A + 1, my_acc[c * 32].y, invQ);
                    } else {
                        add_fixed(A, accRe[c], invQ);
                        add_fixed(A + 1, accIm[c], invQ);
                    }
                }
            }
        }
        if (P.count_stats) {
            cRays = __reduce_add_sync(FULL, cRays);
            cHit = __reduce_add_sync(FULL, cHit);
            cBounce = __reduce_add_sync(FULL, cBounce);
            cQuery = __reduce_add_sync(FULL, cQuery);
            if (lane < 4) {
                const unsigned v = lane == 0 ? cRays : lane == 1 ? cHit : lane == 2 ? cBounce : cQuery;
                if (v) atomicAdd(P.acc_stats + 4 * (size_t)seg + lane, (unsigned long long)v);
            }
        }
    }
    if (err) atomicOr(P.err, err);
}

// ------------------------------------------------------- listed rays (diagnostics)
struct TraceListParams {
    SceneView S;
    const Segment* segs;
    const JobConst* jobs;
    const int32_t* rays;   // [n][3]: segment (angle of the plan's one job), i, j -- checked by the host
    long long n;
    uint32_t* err;
    sbr_ray_record* out;   // [n]
};

// One thread per listed ray: the sweep kernel's own ray start, bounce step and
// finish (ray.cuh), with the record written as k_trace writes it.
template <int PREC>
__global__ void __launch_bounds__(128) k_trace_list(const TraceListParams P) {
    constexpr bool F64 = PREC == SBR_PREC_FP64;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= P.n) return;
    const Segment& G = P.segs[P.rays[3 * t]];
    const JobConst J = P.jobs[G.job];
    const int i = P.rays[3 * t + 1], j = P.rays[3 * t + 2];
    sbr_ray_record* rec = P.out + t;
    uint32_t err = 0;
    RayF rf;
    RayD rd;
    PolF ef;
    PolD ed;
    if (F64) start_d(rd, G, J, i, j);
    else start_f<PREC>(rf, G, J, i, j);
    if (J.max_bounces > 0) {
        bool done = false;
        while (!done)
            done = F64 ? step_d<true, false>(rd, ed, P.S, J.max_bounces, err, rec)
                       : step_f<PREC, true, false>(rf, ef, P.S, J.max_bounces, err, rec, nullptr);
    }
    const RayOut out = F64 ? finish_d(rd, J) : finish_f<PREC>(rf, J);
    rec->count = F64 ? rd.count : rf.count;
    rec->flags = 1;
    rec->dist = out.L;
    if (F64) {
        rec->normal[0] = float(rd.nl.x); rec->normal[1] = float(rd.nl.y); rec->normal[2] = float(rd.nl.z);
        rec->lastdir[0] = float(rd.dl.x); rec->lastdir[1] = float(rd.dl.y); rec->lastdir[2] = float(rd.dl.z);
    } else {
        rec->normal[0] = rf.nl.x; rec->normal[1] = rf.nl.y; rec->normal[2] = rf.nl.z;
        rec->lastdir[0] = rf.dl.x; rec->lastdir[1] = rf.dl.y; rec->lastdir[2] = rf.dl.z;
    }
    if (err) atomicOr(P.err, err);
}

// ------------------------------------------------------- first-hit raster
// Primary rays of one angle are parallel and start at the pixel centres of the
// launcher grid, so the triangles a ray can hit first are those whose projection on
// the launcher plane covers its pixel centre.  The raster bins the triangles to the
// 4x8 ray tiles of the trace (one tile = the block of rays one warp traces) and tests
// each tile's list with the trace's own watertight triangle test, one lane per ray,
// as tile-based rasterisers do:
//   k_tile_bin   lists, per tile, the triangles whose projection (widened by a
//                margin) reaches the rectangle of the tile's pixel centres:
//                projected box first, then the three edges; each tile holds up to
//                `cap` triangles and counts the rest;
//   k_tile_hit   the closest hit of every ray of a tile among its list (the walk's
//                test, nearest t then the tie order), written to the first-hit buffer
//                as a hit key, kZMiss, or kZWalk for a tile with more than `cap`
//                triangles.
// The trace reads each ray's first query from the buffer; every other query walks.
// Mixed precision only: the reference's Moller-Trumbore test of the FP32 mode is not
// watertight, and near grazing incidence its hits can fall outside any margin around
// the triangles' projections.
struct TileParams {
    const GTri* tris;
    const int32_t* tie;            // exact-tie ranks of the scene, or null
    int32_t ntris;
    uint32_t cap;                  // list entries per tile (longer lists: the rays walk)
    const Segment* segs;
    const JobConst* jobs;
    int64_t seg_begin, seg_end;    // the chunk's segments
    int64_t n_tiles;               // the chunk's tiles
    uint32_t* cnt;                 // [n_tiles] triangles that reach each tile
    int32_t* list;                 // [n_tiles * cap] triangle slots
    unsigned long long* zbuf;      // [n_tiles * 32] first-hit entries, tile-major
};
constexpr int kBinThreads = 256;

// Margin (pixels) around a projected triangle: 0.06 pixel plus 2^-19 of the largest
// launcher coordinate over the pixel size, which covers the FP32 rounding of the
// ray origins, of the triangle test's sheared coordinates and of the edge test.
__device__ __forceinline__ double tile_margin(const Segment& G, const JobConst& J) {
    const double ext = fabs(G.llc[0]) + fabs(G.llc[1]) + fabs(G.llc[2]) + fabs(G.u[0]) + fabs(G.u[1]) +
                       fabs(G.u[2]) + fabs(G.v[0]) + fabs(G.v[1]) + fabs(G.v[2]);
    // pixel sizes from FP32 square roots rounded down (only a larger margin results)
    const double pu = double(sqrtf(float(G.u[0] * G.u[0] + G.u[1] * G.u[1] + G.u[2] * G.u[2])) * 0.999999f) / J.nx;
    const double pv = double(sqrtf(float(G.v[0] * G.v[0] + G.v[1] * G.v[1] + G.v[2] * G.v[2])) * 0.999999f) / J.ny;
    return 0.06 + ldexp(ext, -19) / fmin(pu, pv);
}

// A triangle's footprint on one segment's pixel grid: the pixel-centre range of its
// widened projected box (clipped to the segment), the tiles that range spans, and
// its three edges as e(x, y) = ex (x - ilo) + ey (y - jlo) + ec >= 0 inside, in FP32
// about the range's first pixel centre (widened by the margin; a projection of
// near-zero area, or one within two tiles, keeps its box only: ex = ey = 0, ec = 1).
struct TriFoot {
    int ilo, ihi, jlo, jhi;
    int bx0, by0, nbx, ntile;
    int slot;
    float ex[3], ey[3], ec[3];
};
__device__ __forceinline__ int tri_foot(const GTri& T, const Segment& G, double mg, int slot, TriFoot& f) {
    const double X[3] = {T.v0.x, T.v1.x, T.v2.x};
    const double Y[3] = {T.v0.y, T.v1.y, T.v2.y};
    const double Z[3] = {T.v0.z, T.v1.z, T.v2.z};
    double s[3], t[3];
    double smin = 1e300, smax = -1e300, tmin = 1e300, tmax = -1e300;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s[k] = G.ps[0] * X[k] + G.ps[1] * Y[k] + G.ps[2] * Z[k] + G.ps[3];
        t[k] = G.pt[0] * X[k] + G.pt[1] * Y[k] + G.pt[2] * Z[k] + G.pt[3];
        smin = fmin(smin, s[k]); smax = fmax(smax, s[k]);
        tmin = fmin(tmin, t[k]); tmax = fmax(tmax, t[k]);
    }
    // (clamped to [-1, 2e9] before the conversions to int)
    f.ilo = max(G.i0, (int)fmin(fmax(ceil(smin - mg), -1.0), 2.0e9));
    f.ihi = min(G.i0 + G.ni - 1, (int)fmin(fmax(floor(smax + mg), -1.0), 2.0e9));
    f.jlo = max(G.j0, (int)fmin(fmax(ceil(tmin - mg), -1.0), 2.0e9));
    f.jhi = min(G.j0 + G.nj - 1, (int)fmin(fmax(floor(tmax + mg), -1.0), 2.0e9));
    if (f.ihi < f.ilo || f.jhi < f.jlo) return 0;
    f.slot = slot;
    f.bx0 = (f.ilo - G.i0) >> 2;
    f.by0 = (f.jlo - G.j0) >> 3;
    f.nbx = ((f.ihi - G.i0) >> 2) - f.bx0 + 1;
    f.ntile = f.nbx * (((f.jhi - G.j0) >> 3) - f.by0 + 1);
    const double area2 = (s[1] - s[0]) * (t[2] - t[0]) - (t[1] - t[0]) * (s[2] - s[0]);
    const bool edges = f.ntile > 2 && fabs(area2) >= 1e-6;
    const double sg = area2 > 0.0 ? 1.0 : -1.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int n = k == 2 ? 0 : k + 1;
        const double ex = -sg * (t[n] - t[k]), ey = sg * (s[n] - s[k]);
        f.ex[k] = edges ? float(ex) : 0.0f;
        f.ey[k] = edges ? float(ey) : 0.0f;
        // |(ex, ey)| from an FP32 square root rounded up: the margin only widens
        const double len = double(sqrtf(float(ex * ex + ey * ey)) * 1.000001f);
        f.ec[k] = edges ? float(ex * (f.ilo - s[k]) + ey * (f.jlo - t[k]) + mg * len) : 1.0f;
    }
    return f.ntile;
}
// Tile k of the footprint (row-major over its tile range) relative to the
// segment's first tile, or -1 when an edge leaves every pixel centre of the tile
// (inside the footprint's range) outside.
__device__ __forceinline__ int foot_tile(const TriFoot& f, const Segment& G, int k) {
    const int bx = f.bx0 + k % f.nbx, by = f.by0 + k / f.nbx;
    const int x0 = max(G.i0 + kBlockW * bx, f.ilo) - f.ilo, x1 = min(G.i0 + kBlockW * bx + kBlockW - 1, f.ihi) - f.ilo;
    const int y0 = max(G.j0 + kBlockH * by, f.jlo) - f.jlo, y1 = min(G.j0 + kBlockH * by + kBlockH - 1, f.jhi) - f.jlo;
    const float cx = 0.5f * float(x0 + x1), cy = 0.5f * float(y0 + y1);
    const float hx = 0.5f * float(x1 - x0), hy = 0.5f * float(y1 - y0);
#pragma unroll
    for (int e = 0; e < 3; ++e)
        if (f.ex[e] * cx + f.ey[e] * cy + f.ec[e] + fabsf(f.ex[e]) * hx + fabsf(f.ey[e]) * hy < 0.0f) return -1;
    return by * G.blocks_x + bx;
}

// One pass: every lane computes the footprint of its triangle into shared memory,
// then the warp's (triangle, tile) pairs are dealt to its lanes 32 at a time (each
// lane finds its pair's triangle by a binary search over the warp's prefix sums),
// so footprints of any size keep every lane busy.
__global__ void __launch_bounds__(kBinThreads) k_tile_bin(const TileParams P) {
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ TriFoot s_foot[kBinThreads];
    __shared__ int s_pre[kBinThreads];
    const Segment& G = P.segs[P.seg_begin + blockIdx.y];
    if (G.ni <= 0 || G.nj <= 0) return;
    const double mg = tile_margin(G, P.jobs[G.job]);
    const int lane = threadIdx.x & 31;
    TriFoot* const wf = s_foot + (threadIdx.x & ~31);
    int* const wp = s_pre + (threadIdx.x & ~31);
    for (int base = blockIdx.x * blockDim.x; base < P.ntris; base += gridDim.x * blockDim.x) {
        const int slot = base + threadIdx.x;
        int nt = 0;
        if (slot < P.ntris) nt = tri_foot(P.tris[slot], G, mg, slot, wf[lane]);
        int pre = nt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(FULL, pre, off);
            if (lane >= off) pre += y;
        }
        wp[lane] = pre;
        const int total = __shfl_sync(FULL, pre, 31);
        __syncwarp();
        for (int it = lane; it < total; it += 32) {
            int lo = 0, hi = 31;  // the first lane whose inclusive prefix exceeds it
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (wp[mid] > it) hi = mid;
                else lo = mid + 1;
            }
            const TriFoot& f = wf[lo];
            const int b = foot_tile(f, G, it - (lo > 0 ? wp[lo - 1] : 0));
            if (b < 0) continue;
            const int64_t tile = G.tbase + (int64_t)b;
            const uint32_t pos = atomicAdd(P.cnt + tile, 1u);
            if (pos < P.cap) P.list[tile * P.cap + pos] = f.slot;
        }
        __syncwarp();
    }
}

// The closest hit of each lane's ray among a tile's list: 32 triangles at a time,
// each lane loading one (the loads overlap) into the warp's slice of shared memory,
// then every lane testing every triangle (broadcast reads).
template <int KZ>
__device__ __forceinline__ void tile_list_wt(const int32_t* list, uint32_t c, const GTri* tris, const int32_t* tie,
                                             F3 o, const WtRay& w, float& tB, int& best, GTri* s_tri, int* s_slot) {
    const int lane = threadIdx.x & 31;
    for (uint32_t b = 0; b < c; b += 32) {
        const int mine = b + lane < c ? list[b + lane] : 0;
        const GTri M = tris[mine];
        __syncwarp();  // the previous batch is read
        s_tri[lane] = M;
        s_slot[lane] = mine;
        __syncwarp();
        const int n = (int)min(32u, c - b);
        for (int q = 0; q < n; ++q) {
            const int slot = s_slot[q];
            float tt;
            if (wt_tri<KZ>(s_tri[q], o, w, 1.0e-3f, tB, tt) && replaces(tt, slot, tB, best, tie)) {
                tB = tt;
                best = slot;
            }
        }
    }
}

// One warp per tile (grid-stride): every lane's ray starts where the trace starts
// it (primary_origin) and is tested as the trace's first query tests it.
__global__ void __launch_bounds__(256) k_tile_hit(const TileParams P) {
    __shared__ GTri s_tri[256];
    __shared__ int s_slot[256];
    const int lane = threadIdx.x & 31;
    GTri* const wt = s_tri + (threadIdx.x & ~31);
    int* const ws = s_slot + (threadIdx.x & ~31);
    const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < P.n_tiles; t += nw) {
        // the tile's segment: the last of the chunk whose first tile is <= t
        int64_t lo = P.seg_begin, hi = P.seg_end - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) >> 1;
            if (P.segs[mid].tbase <= t) lo = mid;
            else hi = mid - 1;
        }
        const Segment& G = P.segs[lo];
        const uint32_t c = P.cnt[t];
        unsigned long long key = c > P.cap ? kZWalk : kZMiss;
        if (c > 0 && c <= P.cap) {
            const int blk = (int)(t - G.tbase);
            const int i = G.i0 + (blk % G.blocks_x) * kBlockW + (lane % kBlockW);
            const int j = G.j0 + (blk / G.blocks_x) * kBlockH + (lane / kBlockW);
            const F3 o = primary_origin<SBR_PREC_MIXED>(G, P.jobs[G.job], i, j);
            const WtRay w = wt_ray(f3(G.rdf[0], G.rdf[1], G.rdf[2]));
            const int32_t* list = P.list + t * P.cap;
            float tB = 1e20f;
            int best = -1;
            switch (w.kz) {
                case 0: tile_list_wt<0>(list, c, P.tris, P.tie, o, w, tB, best, wt, ws); break;
                case 1: tile_list_wt<1>(list, c, P.tris, P.tie, o, w, tB, best, wt, ws); break;
                default: tile_list_wt<2>(list, c, P.tris, P.tie, o, w, tB, best, wt, ws); break;
            }
            if (best >= 0 && i < G.i0 + G.ni && j < G.j0 + G.nj)
                key = ((unsigned long long)__float_as_uint(tB) << 32) | (unsigned)best;
        }
        P.zbuf[t * 32 + lane] = key;
    }
}

// Converts the fixed-point accumulators (summing the replicas exactly, as
// integers) to fields, copies the counters, and clears accumulators, counters
// and queue heads so the plan can run again without a memset.
__global__ void k_finalize(long long n_samples, int n_rep, const double* __restrict__ quantum,
                           unsigned long long* acc, double* field, long long n_stats,
                           unsigned long long* acc_stats, unsigned long long* out_stats, unsigned long long* queue,
                           long long n_queue) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < n_samples) {
        long long re = 0, im = 0;
        for (int r = 0; r < n_rep; ++r) {
            unsigned long long* A = acc + 2 * (t * n_rep + r);
            re += (long long)A[0];
            im += (long long)A[1];
            A[0] = 0ull;
            A[1] = 0ull;
        }
        const double q = quantum[t];
        field[2 * t] = double(re) * q;
        field[2 * t + 1] = double(im) * q;
    }
    if (t < n_stats) {
        out_stats[t] = acc_stats[t];
        acc_stats[t] = 0ull;
    }
    if (t < n_queue) queue[t] = 0ull;
}

__global__ void k_fill_records(sbr_ray_record* r, long long n) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
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

template <int PREC, int EPI, bool REC, bool POL, bool MULTI, bool W8 = false>
const void* kernel_ptr() {
    return reinterpret_cast<const void*>(&k_trace<PREC, EPI, REC, POL, MULTI, W8>);
}

template <int PREC, bool REC, bool POL, bool MULTI = false>
const void* pick_epi_kernel(int epi) {
    switch (epi) {
        case EPI_LANE1: return kernel_ptr<PREC, EPI_LANE1, REC, POL, MULTI>();
        case EPI_LANE4: return kernel_ptr<PREC, EPI_LANE4, REC, POL, MULTI>();
        case EPI_T64: return kernel_ptr<PREC, EPI_T64, REC, POL, MULTI>();
        default: return kernel_ptr<PREC, EPI_T128, REC, POL, MULTI>();
    }
}

// Trace kernel for a plan: precision, accumulator layout for `channels` (the
// largest frequencies x polarisations of a launch), records, polarisation, and
// whether jobs trace different scenes.  Record kernels come with the two general
// layouts only and one scene; polarised kernels in MIXED and FP64 precision only
// (the host rejects the other combinations).
const void* pick_kernel(int prec, int channels, bool rec, bool pol, bool multi = false, bool w8 = false) {
    int epi = pick_epi(channels);
    if (w8 && prec == SBR_PREC_MIXED && !rec && !pol && !multi) {
        switch (epi) {
            case EPI_LANE1: return kernel_ptr<SBR_PREC_MIXED, EPI_LANE1, false, false, false, true>();
            case EPI_LANE4: return kernel_ptr<SBR_PREC_MIXED, EPI_LANE4, false, false, false, true>();
            case EPI_T64: return kernel_ptr<SBR_PREC_MIXED, EPI_T64, false, false, false, true>();
            default: return kernel_ptr<SBR_PREC_MIXED, EPI_T128, false, false, false, true>();
        }
    }
    if (multi && !rec) {
        if (pol) return prec == SBR_PREC_FP64 ? pick_epi_kernel<SBR_PREC_FP64, false, true, true>(epi)
                                              : pick_epi_kernel<SBR_PREC_MIXED, false, true, true>(epi);
        switch (prec) {
            case SBR_PREC_MIXED: return pick_epi_kernel<SBR_PREC_MIXED, false, false, true>(epi);
            case SBR_PREC_FP32: return pick_epi_kernel<SBR_PREC_FP32, false, false, true>(epi);
            default: return pick_epi_kernel<SBR_PREC_FP64, false, false, true>(epi);
        }
    }
    if (rec) {
        epi = epi <= EPI_LANE4 ? EPI_LANE4 : EPI_T128;
        switch (prec) {
            case SBR_PREC_MIXED: return pick_epi_kernel<SBR_PREC_MIXED, true, false>(epi);
            case SBR_PREC_FP32: return pick_epi_kernel<SBR_PREC_FP32, true, false>(epi);
            default: return pick_epi_kernel<SBR_PREC_FP64, true, false>(epi);
        }
    }
    if (pol) return prec == SBR_PREC_FP64 ? pick_epi_kernel<SBR_PREC_FP64, false, true>(epi)
                                          : pick_epi_kernel<SBR_PREC_MIXED, false, true>(epi);
    switch (prec) {
        case SBR_PREC_MIXED: return pick_epi_kernel<SBR_PREC_MIXED, false, false>(epi);
        case SBR_PREC_FP32: return pick_epi_kernel<SBR_PREC_FP32, false, false>(epi);
        default: return pick_epi_kernel<SBR_PREC_FP64, false, false>(epi);
    }
}

sbr_status launch_trace(const void* fn, int grid, cudaStream_t st, const TraceParams& p) {
    void* args[] = {const_cast<TraceParams*>(&p)};
    SBR_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(kCtaThreads), args, 0, st));
    return SBR_OK;
}

sbr_status resident_ctas(const void* fn, int ctas_per_sm, int num_sms, int* out) {
    int occ = 0;
    SBR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kCtaThreads, 0));
    *out = std::max(1, ctas_per_sm > 0 ? ctas_per_sm : occ) * num_sms;
    return SBR_OK;
}

void finalize(long long n_samples, int n_rep, const double* quantum, unsigned long long* acc, double* field,
              long long n_stats, unsigned long long* acc_stats, unsigned long long* out_stats,
              unsigned long long* queue, long long n_queue, cudaStream_t st) {
    long long nmax = std::max(std::max(n_samples, n_stats), std::max(n_queue, 1LL));
    k_finalize<<<(unsigned)((nmax + 255) / 256), 256, 0, st>>>(n_samples, n_rep, quantum, acc, field, n_stats,
                                                               acc_stats, out_stats, queue, n_queue);
}

}  // namespace

namespace {

// Bins and rasterises the first hits of one chunk into the first-hit buffer.
sbr_status tile_raster(sbr_plan* pl, const sbr_plan::Chunk& ch, cudaStream_t st, int& launches) {
    TileParams t{};
    t.tris = pl->scene_view.tris;
    t.tie = pl->scene_view.tie;
    t.ntris = (int32_t)pl->scene->ntris;
    t.cap = pl->tile_cap;
    t.segs = pl->d_segs;
    t.jobs = pl->d_jobs;
    t.seg_begin = ch.seg_begin;
    t.seg_end = ch.seg_end;
    t.n_tiles = ch.tiles;
    t.cnt = pl->d_tile_cnt;
    t.list = pl->d_tile_list;
    t.zbuf = pl->d_zbuf;
    SBR_CUDA(cudaMemsetAsync(t.cnt, 0, (size_t)t.n_tiles * sizeof(uint32_t), st));
    const unsigned gx = (unsigned)std::min<long long>((t.ntris + kBinThreads - 1) / kBinThreads, 4096);
    k_tile_bin<<<dim3(gx, (unsigned)(t.seg_end - t.seg_begin)), kBinThreads, 0, st>>>(t);
    const unsigned gh = (unsigned)std::min<long long>((t.n_tiles + 7) / 8, (long long)pl->num_sms * 64);
    k_tile_hit<<<gh, 256, 0, st>>>(t);
    launches += 2;
    SBR_CUDA(cudaGetLastError());
    return SBR_OK;
}

}  // namespace

sbr_status plan_launch(sbr_plan* pl, bool records, sbr_ray_record* d_records) {
    const bool pol = pl->pol == SBR_POL_HHVV && !records;
    const int npol = pol ? 2 : 1;
    const bool batched = pl->mode == SBR_MODE_BATCHED || records;
    const void* fn = pick_kernel(pl->prec, (batched ? pl->k_max : 1) * npol, records, pol, pl->multi,
                                 pl->scene_view.nodes8 != nullptr);
    TraceParams p{};
    p.segpol = pl->d_segpol;
    p.scenes = pl->d_scenes;
    p.S = pl->scene_view;
    p.segs = pl->d_segs;
    p.seg_item_base = pl->d_seg_base;
    p.n_segs = (int32_t)pl->n_segs;
    p.n_rep = kAccReplicas;
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
        if (pl->persistent_grid <= 0) {
            sbr_status s = resident_ctas(fn, pl->ctas_per_sm, pl->num_sms, &pl->persistent_grid);
            if (s != SBR_OK) return s;
        }
        if ((pl->mode == SBR_MODE_BATCHED || records) && pl->raster) {
            // per chunk of segments: first hits by the tile raster, then the persistent trace
            p.k_begin = 0;
            p.k_count = 0;
            p.count_stats = 1;
            p.zbuf = pl->d_zbuf;
            p.tile_cnt = pl->d_tile_cnt;
            for (size_t c = 0; c < pl->chunks.size(); ++c) {
                const sbr_plan::Chunk& ch = pl->chunks[c];
                if (ch.tiles > 0) {
                    sbr_status s = tile_raster(pl, ch, st, launches);
                    if (s != SBR_OK) return s;
                }
                if (ch.item_end > ch.item_begin) {
                    p.item_begin = ch.item_begin;
                    p.item_end = ch.item_end;
                    p.queue = pl->d_queue + 1 + pl->n_samples + c;
                    const int grid = (int)std::min<long long>(pl->persistent_grid, (ch.item_end - ch.item_begin + 3) / 4);
                    sbr_status s = launch_trace(fn, grid, st, p);
                    if (s != SBR_OK) return s;
                    ++launches;
                }
            }
        } else if (pl->mode == SBR_MODE_BATCHED || records) {
            p.k_begin = 0;
            p.k_count = 0;
            p.count_stats = 1;
            p.item_begin = 0;
            p.item_end = pl->n_items;
            p.queue = pl->d_queue;
            const long long warps_needed = pl->n_items;
            const int grid = (int)std::min<long long>(pl->persistent_grid, (warps_needed + 3) / 4);
            sbr_status s = launch_trace(fn, grid, st, p);
            if (s != SBR_OK) return s;
            ++launches;
        } else {
            // the reference loop: one trace + PO launch per (angle, frequency), each
            // with its own queue head
            for (size_t g = 0; g < pl->segs.size(); ++g) {
                const Segment& G = pl->segs[g];
                const long long n = pl->seg_base[g + 1] - pl->seg_base[g];
                if (n == 0) continue;
                const JobConst& J = pl->jobs[G.job];
                for (int k = 0; k < J.n_freqs; ++k) {
                    p.k_begin = k;
                    p.k_count = 1;
                    p.count_stats = k == 0;
                    p.item_begin = pl->seg_base[g];
                    p.item_end = pl->seg_base[g + 1];
                    p.queue = pl->d_queue + 1 + G.sample_base + k;
                    const int grid = (int)std::min<long long>(pl->persistent_grid, (n + 3) / 4);
                    sbr_status s = launch_trace(fn, grid, st, p);
                    if (s != SBR_OK) return s;
                    ++launches;
                }
            }
        }
    }
    finalize(pl->n_samples * npol, kAccReplicas, pl->d_quantum, pl->d_acc, pl->d_field, (long long)pl->n_segs * 4,
             pl->d_acc_stats, pl->d_stats, pl->d_queue, pl->n_samples + 1 + (long long)pl->chunks.size(), st);
    SBR_CUDA(cudaGetLastError());
    ++launches;
    pl->launches = launches;
    return SBR_OK;
}

sbr_status trace_list_launch(sbr_plan* pl, const int32_t* d_rays, long long n, sbr_ray_record* d_out) {
    if (n <= 0) return SBR_OK;
    TraceListParams p{};
    p.S = pl->scene_view;
    p.segs = pl->d_segs;
    p.jobs = pl->d_jobs;
    p.rays = d_rays;
    p.n = n;
    p.err = pl->d_err;
    p.out = d_out;
    const void* fn = pl->prec == SBR_PREC_FP64   ? reinterpret_cast<const void*>(&k_trace_list<SBR_PREC_FP64>)
                     : pl->prec == SBR_PREC_FP32 ? reinterpret_cast<const void*>(&k_trace_list<SBR_PREC_FP32>)
                                                 : reinterpret_cast<const void*>(&k_trace_list<SBR_PREC_MIXED>);
    void* args[] = {&p};
    SBR_CUDA(cudaLaunchKernel(fn, dim3((unsigned)((n + 127) / 128)), dim3(128), args, 0, pl->stream));
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
    if (o.polarization != SBR_POL_SCALAR)
        return fail(SBR_ERR_UNSUPPORTED, "the allocation-free sweep computes the scalar field only");
    sbr_status st = validate_run(s, job, 1, o);
    if (st != SBR_OK) return st;
    if (job->n_angles > SBR_NOALLOC_MAX_ANGLES)
        return fail(SBR_ERR_TOO_LARGE, "allocation-free sweep: more than SBR_NOALLOC_MAX_ANGLES (1024) angles");
    if (job->n_angles * job->n_freqs > SBR_NOALLOC_MAX_SAMPLES)
        return fail(SBR_ERR_TOO_LARGE, "allocation-free sweep: more than SBR_NOALLOC_MAX_SAMPLES (4096) samples");
    if (o.precision == SBR_PREC_FP64 && !s->d_tris64)
        return fail(SBR_ERR_UNSUPPORTED, "allocation-free FP64 sweep needs a scene created with want_fp64 = 1");

    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    sbr::DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(s->device));
    NoallocScratch* D = nullptr;
    st = noalloc_address(s->device, &D);
    if (st != SBR_OK) return st;

    NoallocSink sink;
    g_noalloc_host.seg_base[0] = 0;
    TableTotals tot;
    const sbr_scene* one[1] = {s};
    st = build_tables(one, nullptr, job, 1, o, sink, tot);
    if (st != SBR_OK) return st;

    cudaStream_t stream = o.stream ? (cudaStream_t)o.stream : s->stream;
    // From the first queued copy on, every return waits for this call's work on the
    // shared array, so the next call (after the lock is released) cannot overlap it.
    struct StreamDrain {
        cudaStream_t st;
        ~StreamDrain() { cudaStreamSynchronize(st); }
    } drain{stream};
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
        const void* fn = pick_kernel(o.precision, tot.k_max, false, false);
        int resident = 0;
        st = resident_ctas(fn, o.ctas_per_sm, s->num_sms, &resident);
        if (st != SBR_OK) return st;
        TraceParams p{};
        p.S = s->view();
        p.segs = D->tables.segs;
        p.seg_item_base = D->tables.seg_base;
        p.n_segs = (int32_t)nseg;
        p.k_begin = 0;
        p.k_count = 0;
        p.count_stats = 1;
        p.n_rep = 1;
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
        const int grid = (int)std::min<long long>(resident, (tot.n_items + 3) / 4);
        st = launch_trace(fn, grid, stream, p);
        if (st != SBR_OK) return st;
    }
    finalize((long long)nsamp, 1, D->tables.quantum, D->acc, d_field, d_stats ? 4LL * (long long)nseg : 0LL,
             D->acc_stats, reinterpret_cast<unsigned long long*>(d_stats), &D->queue, 1, stream);
    SBR_CUDA(cudaGetLastError());
    SBR_CUDA(cudaStreamSynchronize(stream));

    uint32_t e = 0;
    SBR_CUDA(cudaMemcpy(&e, s->d_err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) clear_device_word(s->d_err);
    if (e & DEV_ERR_CANCEL) return fail(SBR_ERR_CANCELLED, "run cancelled");
    if (e & DEV_ERR_BUDGET) return fail(SBR_ERR_TIMEOUT, "traversal iteration budget exceeded");
    if (e & DEV_ERR_STACK) return fail(SBR_ERR_STACK, "traversal stack overflow");
    return SBR_OK;
}
