// errbound.cu -- sbr_error_bound: the error, per (angle, frequency) sample, of the
// mixed-precision sweep (FP32 traversal, FP64 path, FP32 phase pairs, FP64 sums of
// FP32 block partials) against the FP64 sweep of the same job.  No counterpart in the reference, which has no
// mixed-precision mode.
//
// A second pass re-traces every ray of the plan with the mixed sweep's own
// arithmetic (start_f and the step of ray.cuh, the watertight test of trace.cuh:
// the same hits bit for bit) while carrying bounds on how far the FP32 ray can be
// from the FP64 ray with the same hits:
//   e   position error across the ray (m): origin rounding, then per bounce the
//       lateral drift t * a, the induced change of t and the FP32 roundings;
//   a   direction error (rad): rounding of -dir, then per reflection twice the
//       error of the FP32 normal (8 u / sin of the triangle's corner angle) + 4 u;
//   dL  path-length error (m): per bounce (e + t a) / |cos i| + 4 u t.
// A ray is re-traced in FP64 when one of its decisions lies within that
// uncertainty of flipping -- a tested triangle whose edge lies within 2 (e + a D)
// of the ray (hit or miss; D = scene diagonal, 2 covers the oblique projection of
// the sheared test), |det| within a factor 2 of the 1e-6 threshold, t within
// dt = 4 m + 4 u (|o| + D) of tMin or of the current closest hit -- or when its
// phase uncertainty 2 k_max dL exceeds 0.05 rad.  Boxes are widened by the same
// margin during this pass, so a near miss inside a culled box is still tested
// (boxes only prune; the closest hit does not change).  For those rays the exact
// difference of the FP64 and mixed terms is summed per sample (Delta_k).  The other
// rays differ from FP64 only by rounding, |d term| <= scale_k (amp 2 k dL + amp eps
// + damp), damp = 2 R^n (dn_last + a).  Part of those errors is the same for every
// ray that sees the same geometry the same way (a face-on plate): the relative error
// of t from the approximate reciprocals of the triangle test (bounded by 8 u t per
// bounce, dLs) and the error of the sine / cosine approximation (eps).  That shared
// part adds coherently, so it is bounded by the field itself times its
// amp-weighted mean, |S_k| (2 k c1 + eps) with c1 = sum amp dLs / sum amp.  The rest
// (origin, hit-point and direction rounding) varies from ray to ray as independent,
// zero-mean errors, bounded with the probabilistic rounding-error bound of Higham
// and Mary (SIAM J. Sci. Comput. 41(5), 2019): |sum| <= lambda sqrt(sum of squares),
// exceeded with probability below 4 exp(-lambda^2 / 2) (lambda = 6: 6e-8).  Per
// sample
//   E_k = |Delta_k| + |S_k| (2 k c1 + eps) + lambda scale_k (2 k sqrt(Q1) + sqrt(Q0))
//         + (items + 1) quantum_k,
//         + lambda scale_k u sqrt(Q2),
// Q1 = sum (amp (dL - dLs))^2, Q0 = sum damp^2 over the rounding-only rays; the
// fixed-point term covers the fixed-point fold of the sweep.  The last term covers
// the FP32 partial sums of the lane-owned epilogue: each term of a 4x8 ray block is
// added to its channel's FP32 partial by one FMA, rounded within u |partial|, and
// every partial is within A_b = sum |amp| of the block, so Q2 = sum over blocks of
// n_b A_b^2 (n_b terms); the per-lane layouts sum in FP64 and the term only
// overstates their error.  The phase pair's 2^-45 |x| turns (ray.cuh, turns_frac)
// is added to dLs as 2^-45 L.
#include <algorithm>
#include <cmath>
#include <vector>

#include "plan.hpp"
#include "ray.cuh"

namespace sbr {
namespace {

constexpr float kU = 5.9604644775390625e-08f;  // 2^-24, unit roundoff of FP32
// Phase / amplitude error of one mixed term: the rounding of the FP32 remainder of
// 2 k L in turns (2 pi 2^-25 rad; the FP32 pair's 2^-45 |x| is carried in dLs),
// __sincosf (below 4e-7 absolute), FP32 amplitude (2^-24).
constexpr double kPhaseEps = 1.0e-6;

constexpr double kPhaseExact = 0.05;  // rad: rays with more phase uncertainty are re-traced in FP64
constexpr double kLambda = 6.0;       // probabilistic bound multiplier (failure below 6e-8)

struct ErrParams {
    SceneView S;
    const Segment* segs;
    const int64_t* seg_item_base;
    int32_t n_segs;
    const JobConst* jobs;
    const FreqConst* freqs;
    int64_t n_items;
    unsigned long long* queue;
    double* acc;       // [n_segs][8]: sum amp, sum amp dLs, Q2, Q1, Q0, re-traced rays, rays, -
    double* dfield;    // [n_samples][2]: sum of (FP64 term - mixed term) of the re-traced rays
    float diag;        // scene bounding-box diagonal (m)
    uint32_t* err;
    const volatile int32_t* cancel;
};

__device__ __forceinline__ float norm1(F3 v) { return fabsf(v.x) + fabsf(v.y) + fabsf(v.z); }

// The watertight test of trace.cuh (wt_tri, identical decisions), flagging in `amb`
// a decision within the margin m (edges) / dt (t) of flipping.
template <int KZ>
__device__ __forceinline__ bool wt_tri_flag(const GTri& T, F3 o, const WtRay& w, float tMin, float tMax, float m,
                                            float dt, float& t, bool& amb) {
    constexpr int KX = (KZ + 1) % 3, KY = (KZ + 2) % 3;
    const float ox = axis<KX>(o), oy = axis<KY>(o), oz = axis<KZ>(o);
    const float az = __fsub_rn(axis<KZ>(T.v0), oz), bz = __fsub_rn(axis<KZ>(T.v1), oz),
                cz = __fsub_rn(axis<KZ>(T.v2), oz);
    const float ax = __fmaf_rn(-w.sx, az, __fsub_rn(axis<KX>(T.v0), ox));
    const float ay = __fmaf_rn(-w.sy, az, __fsub_rn(axis<KY>(T.v0), oy));
    const float bx = __fmaf_rn(-w.sx, bz, __fsub_rn(axis<KX>(T.v1), ox));
    const float by = __fmaf_rn(-w.sy, bz, __fsub_rn(axis<KY>(T.v1), oy));
    const float cx = __fmaf_rn(-w.sx, cz, __fsub_rn(axis<KX>(T.v2), ox));
    const float cy = __fmaf_rn(-w.sy, cz, __fsub_rn(axis<KY>(T.v2), oy));
    float U = __fsub_rn(__fmul_rn(cx, by), __fmul_rn(cy, bx));
    float V = __fsub_rn(__fmul_rn(ax, cy), __fmul_rn(ay, cx));
    float W = __fsub_rn(__fmul_rn(bx, ay), __fmul_rn(by, ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = float(__dsub_rn(__dmul_rn(cx, by), __dmul_rn(cy, bx)));
        V = float(__dsub_rn(__dmul_rn(ax, cy), __dmul_rn(ay, cx)));
        W = float(__dsub_rn(__dmul_rn(bx, ay), __dmul_rn(by, ax)));
    }
    const bool inside = !((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f));
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    // margins: distance (sheared plane) from the ray to each edge line, and t of the plane
    const float dU = fabsf(U) * rhypotf(cx - bx, cy - by), dV = fabsf(V) * rhypotf(ax - cx, ay - cy),
                dW = fabsf(W) * rhypotf(bx - ax, by - ay);
    const float T3 = __fmaf_rn(U, az, __fmaf_rn(V, bz, __fmul_rn(W, cz)));
    const float tp = det != 0.0f ? T3 * w.sz / det : 0.0f;
    const bool inRange = tp >= tMin - dt && tp <= tMax + dt;
    if (inRange) {
        if (inside) {
            if (fminf(dU, fminf(dV, dW)) < m) amb = true;
        } else {
            // the ray is outside across the edges whose function disagrees with the
            // orientation; it would be inside if each of those moved by less than m
            const bool pos = det >= 0.0f;
            const bool vU = pos ? U < 0.0f : U > 0.0f, vV = pos ? V < 0.0f : V > 0.0f, vW = pos ? W < 0.0f : W > 0.0f;
            if ((!vU || dU < m) && (!vV || dV < m) && (!vW || dW < m)) amb = true;
        }
        const float adet = fabsf(det) * w.adz;
        if (adet >= 0.5e-6f && adet < 2.0e-6f) amb = true;
    }
    if (!inside) return false;
    if (!(fabsf(det) * w.adz >= 1.0e-6f)) return false;
    float rdet;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rdet) : "f"(det));
    const float tt = __fmul_rn(__fmul_rn(T3, w.sz), rdet);
    if (fabsf(tt - tMin) < dt || fabsf(tt - tMax) < dt) amb = true;
    if (!(tt >= tMin && tt <= tMax)) return false;
    t = tt;
    return true;
}

template <int KZ>
__device__ __forceinline__ void leaf_flag(const GTri* __restrict__ tris, const int32_t* tie, int first, int cnt, F3 o,
                                          const WtRay& w, float tMin, float m, float dt, float& tBest, int& best,
                                          bool& amb) {
    for (int k = 0; k < cnt; ++k) {
        float tt;
        if (wt_tri_flag<KZ>(tris[first + k], o, w, tMin, tBest, m, dt, tt, amb) &&
            replaces(tt, first + k, tBest, best, tie)) {
            tBest = tt;
            best = first + k;
        }
    }
}

// Closest hit as Walker<false> finds it (4-wide nodes, watertight test), with every
// box widened by m across the ray and dt along it, and decisions near flipping
// flagged in `amb`.
__device__ int closest_flag(const SceneView& S, F3 o, F3 d, float tMin, float& tBest, float m, float dt, bool& amb,
                            uint32_t& err) {
    const F3 inv{slab_inv(d.x), slab_inv(d.y), slab_inv(d.z)};
    const WtRay wr = wt_ray(d);
    const F3 oi{o.x * inv.x, o.y * inv.y, o.z * inv.z};
    const float px = m * fabsf(inv.x), py = m * fabsf(inv.y), pz = m * fabsf(inv.z);
    const unsigned onx = inv.x < 0.0f ? 16u : 0u, ony = inv.y < 0.0f ? 48u : 32u, onz = inv.z < 0.0f ? 80u : 64u;
    const unsigned ofx = onx ^ 16u, ofy = ony ^ 16u, ofz = onz ^ 16u;
    unsigned long long stack[kStackDepth];
    int sp = 0, ref = 0, best = -1;
    uint32_t iters = 0;
    auto plane = [](const GNode4* p, unsigned off) {
        return __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const char*>(p) + off));
    };
    auto slab = [&](float nx, float fx, float ny, float fy, float nz, float fz, bool& hit) {
        const float tn = max3f(fmaf(nx, inv.x, -oi.x) - px, fmaf(ny, inv.y, -oi.y) - py,
                               fmaxf(fmaf(nz, inv.z, -oi.z) - pz, tMin - dt));
        const float tf = min3f(fmaf(fx, inv.x, -oi.x) + px, fmaf(fy, inv.y, -oi.y) + py,
                               fminf(fmaf(fz, inv.z, -oi.z) + pz, tBest + dt));
        hit = tn <= tf * kSlabSlack;
        return tn;
    };
    for (;;) {
        while (ref >= 0) {
            if (++iters > kIterBudget) { err |= DEV_ERR_BUDGET; return -1; }
            const GNode4* np = S.nodes + ref;
            const float4 nx = plane(np, onx), fx = plane(np, ofx), ny = plane(np, ony), fy = plane(np, ofy);
            const float4 nz = plane(np, onz), fz = plane(np, ofz);
            const int4 ch = __ldg(&np->child);
            bool h[4];
            float t[4] = {slab(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, h[0]), slab(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, h[1]),
                          slab(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, h[2]), slab(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, h[3])};
            int c[4] = {ch.x, ch.y, ch.z, ch.w};
            const float inf = __int_as_float(0x7f800000);
            for (int k = 0; k < 4; ++k) t[k] = h[k] ? t[k] : inf;
            sort4(t, c);
            for (int k = 3; k >= 0; --k)
                if (t[k] != inf) {
                    if (sp < kStackDepth) stack[sp++] = pack_entry(c[k], t[k]);
                    else err |= DEV_ERR_STACK;
                }
            ref = -1;
            while (sp > 0) {
                const unsigned long long e = stack[--sp];
                if (__uint_as_float((unsigned)(e >> 32)) <= tBest + dt) { ref = (int)(unsigned)e; break; }
            }
            if (ref == -1) return best;
            while (ref < 0) {
                if (++iters > kIterBudget) { err |= DEV_ERR_BUDGET; return -1; }
                const int code = ~ref;
                const int first = code >> 4, cnt = code & 15;
                switch (wr.kz) {
                    case 0: leaf_flag<0>(S.tris, S.tie, first, cnt, o, wr, tMin, m, dt, tBest, best, amb); break;
                    case 1: leaf_flag<1>(S.tris, S.tie, first, cnt, o, wr, tMin, m, dt, tBest, best, amb); break;
                    default: leaf_flag<2>(S.tris, S.tie, first, cnt, o, wr, tMin, m, dt, tBest, best, amb); break;
                }
                ref = -1;
                while (sp > 0) {
                    const unsigned long long e = stack[--sp];
                    if (__uint_as_float((unsigned)(e >> 32)) <= tBest + dt) { ref = (int)(unsigned)e; break; }
                }
                if (ref == -1) return best;
            }
        }
    }
}

// One ray: the mixed sweep's path (start_f, then step_f's arithmetic per bounce)
// with the uncertainty bounds carried along; rays near a decision or with a large
// phase uncertainty are re-traced with the FP64 sweep's own step and their term
// differences added to dfield, the others add to the lane's sums of squares.
// Returns the amplitude the sweep adds for the ray (0 when it adds nothing).
__device__ __forceinline__ float ray_bound(const ErrParams& P, const Segment& G, const JobConst& J, const FreqConst* F,
                                         int K, double kmax, int i, int j, double& sa, double& s1, double& q1,
                                         double& s0, unsigned& nex, uint32_t& err) {
    RayF r;
    start_f<SBR_PREC_MIXED>(r, G, J, i, j);
    float ue = 2.0f * kU * norm1(r.o);  // origin formed in FP64, rounded to FP32
    float ua = 2.0f * kU;                // FP32 direction
    double dL = double(kU * norm1(r.o));
    double dLs = 0.0;  // the part shared by rays seeing the same geometry the same way
    float dnl = 0.0f;
    bool amb = false;
    for (int b = 0; b < J.max_bounces; ++b) {
        // a ray already bound for the FP64 re-trace needs no more margins: it walks
        // unpadded (its uncertainty can grow to metres after a grazing bounce, and
        // boxes widened that far would open most of the tree)
        const bool exact = amb || 2.0 * kmax * dL > kPhaseExact;
        const float m = exact ? 0.0f : 2.0f * (ue + ua * P.diag);
        const float dt = exact ? 0.0f : 4.0f * m + 4.0f * kU * (norm1(r.o) + P.diag);
        float tB = 1e20f;
        const int slot = closest_flag(P.S, r.o, r.d, 1.0e-3f, tB, m, dt, amb, err);
        if (slot < 0) break;
        const GTri T = P.S.tris[slot];
        const F3 n = f3(T.v0.w, T.v1.w, T.v2.w);
        // the step of step_f (ray.cuh), operation for operation
        r.cosl = dot(n, f3(-r.d.x, -r.d.y, -r.d.z));
        r.nl = n;
        r.dl = r.d;
        ++r.count;
        r.L += double(tB);
        const F3 p = fma3(tB, r.d, r.o);
        r.d = reflect_dir(r.d, n);
        r.o = nudge(p, n);
        // uncertainty of this bounce
        const F3 e1 = f3(T.v1.x - T.v0.x, T.v1.y - T.v0.y, T.v1.z - T.v0.z);
        const F3 e2 = f3(T.v2.x - T.v0.x, T.v2.y - T.v0.y, T.v2.z - T.v0.z);
        const F3 N = cross(e1, e2);
        const float sinang = sqrtf(dot(N, N) / fmaxf(dot(e1, e1) * dot(e2, e2), 1e-30f));
        const float dnrm = 8.0f * kU / fmaxf(sinang, 1e-6f);
        const float ci = fmaxf(fabsf(r.cosl), 1e-6f);
        const float dtb = (ue + tB * ua) / ci + 8.0f * kU * tB;
        dL += double(dtb);
        dLs += double(8.0f * kU * tB);
        ue = ue + tB * ua + dtb + 2.0f * kU * norm1(p) + 1.0e-4f * dnrm;
        ua = ua + 2.0f * dnrm + 4.0f * kU;
        dnl = dnrm;
    }
    const RayOut om = finish_f<SBR_PREC_MIXED>(r, J);
    dLs += ldexp(om.L, -45);  // the FP32 phase pair (ray.cuh, turns_frac)
    dL += ldexp(om.L, -45);
    if (amb || (r.count > 0 && 2.0 * kmax * dL > kPhaseExact)) {
        // the FP64 sweep's own ray (start_d / step_d) and the exact term differences
        RayD rd;
        PolD ed;
        start_d(rd, G, J, i, j);
        if (J.max_bounces > 0) {
            bool done = false;
            while (!done) done = step_d<false, false>(rd, ed, P.S, J.max_bounces, err, nullptr);
        }
        const RayOut od = finish_d(rd, J);
        for (int k = 0; k < K; ++k) {
            double re = 0.0, im = 0.0, rm = 0.0, imm = 0.0;
            if (od.amp != 0.0f) po_term(SBR_PREC_FP64, F[k], od, re, im);
            if (om.amp != 0.0f) po_term(SBR_PREC_MIXED, F[k], om, rm, imm);
            re -= rm * F[k].scale;  // mixed terms are summed without k A / (4 pi)
            im -= imm * F[k].scale;
            if (re != 0.0 || im != 0.0) {
                atomicAdd(P.dfield + 2 * (G.sample_base + k), re);
                atomicAdd(P.dfield + 2 * (G.sample_base + k) + 1, im);
            }
        }
        ++nex;
    } else if (r.count > 0) {
        sa += double(om.amp);
        s1 += double(om.amp) * dLs;
        const double e1 = double(om.amp) * (dL - dLs), e0 = 2.0 * double(fabsf(om.Rn)) * double(dnl + ua);
        q1 += e1 * e1;
        s0 += e0 * e0;
    }
    return om.amp;
}

__global__ void __launch_bounds__(kCtaThreads) k_errbound(const ErrParams P) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    uint32_t err = 0;
    for (;;) {
        long long item = 0;
        if (lane == 0) {
            item = (long long)atomicAdd(P.queue, 1ull);
            if (item < P.n_items && P.cancel && *P.cancel != 0) {
                atomicOr(P.err, DEV_ERR_CANCEL);
                item = P.n_items;
            }
        }
        item = __shfl_sync(FULL, item, 0);
        if (item >= P.n_items) break;
        const int seg = find_segment(P.seg_item_base, P.n_segs, item);
        const Segment& G = P.segs[seg];
        const JobConst J = P.jobs[G.job];
        const FreqConst* F = P.freqs + J.freq_base;
        double kmax = 0.0;
        for (int k = 0; k < J.n_freqs; ++k) kmax = fmax(kmax, F[k].k);
        const int b0 = int(item - G.item_base) * G.blocks_per_item;
        const int b1 = min(b0 + G.blocks_per_item, G.blocks);
        double sa = 0.0, s1 = 0.0, q1 = 0.0, s0 = 0.0, q2 = 0.0;
        unsigned nex = 0, nray = 0;
        for (int blk = b0; blk < b1; ++blk) {
            const int i = G.i0 + (blk % G.blocks_x) * kBlockW + (lane % kBlockW);
            const int j = G.j0 + (blk / G.blocks_x) * kBlockH + (lane / kBlockW);
            float am = 0.0f;
            if (i < G.i0 + G.ni && j < G.j0 + G.nj) {
                am = ray_bound(P, G, J, F, J.n_freqs, kmax, i, j, sa, s1, q1, s0, nex, err);
                ++nray;
            }
            // the block's FP32 partial sums: n_b terms, every partial within A_b
            double ab = double(fabsf(am));
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) ab += __shfl_xor_sync(FULL, ab, off);
            const int nb = __popc(__ballot_sync(FULL, am != 0.0f));
            if (lane == 0) q2 += double(nb) * ab * ab;
        }
        for (int off = 16; off > 0; off >>= 1) {
            sa += __shfl_xor_sync(FULL, sa, off);
            s1 += __shfl_xor_sync(FULL, s1, off);
            q1 += __shfl_xor_sync(FULL, q1, off);
            s0 += __shfl_xor_sync(FULL, s0, off);
            q2 += __shfl_xor_sync(FULL, q2, off);
        }
        nex = __reduce_add_sync(FULL, nex);
        nray = __reduce_add_sync(FULL, nray);
        if (lane == 0) {
            double* A = P.acc + 8 * seg;
            atomicAdd(A, sa);
            atomicAdd(A + 1, s1);
            atomicAdd(A + 2, q2);
            atomicAdd(A + 3, q1);  // sums of squares of independent per-ray bounds
            atomicAdd(A + 4, s0);
            atomicAdd(A + 5, double(nex));
            atomicAdd(A + 6, double(nray));
        }
    }
    if (err) atomicOr(P.err, err);
}

}  // namespace
}  // namespace sbr

extern "C" sbr_status sbr_error_bound(sbr_scene* s, const sbr_job* jobs, size_t n_jobs, const sbr_run_opts* opts,
                                      const double* field, double* err_field, double* err_db) {
    using namespace sbr;
    if (!s || (!jobs && n_jobs) || !field) return fail(SBR_ERR_INVALID_ARG, "scene, jobs and field are required");
    sbr_run_opts o{};
    if (opts) o = *opts;
    if (o.precision != SBR_PREC_MIXED)
        return fail(SBR_ERR_UNSUPPORTED, "the error bound is stated for SBR_PREC_MIXED results");
    if (o.polarization != SBR_POL_SCALAR) return fail(SBR_ERR_UNSUPPORTED, "the error bound covers the scalar field");
    o.mode = SBR_MODE_BATCHED;
    o.first_hit = SBR_FIRST_HIT_TRAVERSE;
    o.use_graph = 0;
    o.autotune = 0;
    DeviceGuard device_guard;
    SBR_CUDA(cudaSetDevice(s->device));
    sbr_status st = ensure_fp64(s);  // the re-traced rays walk the FP64 triangles
    if (st != SBR_OK) return st;
    sbr_plan* p = nullptr;
    st = sbr_plan_create(s, jobs, n_jobs, &o, &p);
    if (st != SBR_OK) return st;
    double* d_acc = nullptr;
    double* d_dfield = nullptr;
    unsigned long long* d_queue = nullptr;
    std::vector<double> acc(8 * (size_t)std::max<int64_t>(p->n_segs, 1), 0.0);
    std::vector<double> dfield(2 * (size_t)std::max<int64_t>(p->n_samples, 1), 0.0);
    cudaError_t e = cudaMalloc(&d_acc, acc.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_dfield, dfield.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_queue, sizeof(unsigned long long));
    if (e != cudaSuccess) st = fail(SBR_ERR_OOM, "error-bound accumulators");
    if (st == SBR_OK) {
        e = cudaMemsetAsync(d_acc, 0, acc.size() * sizeof(double), p->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_dfield, 0, dfield.size() * sizeof(double), p->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned long long), p->stream);
        if (e != cudaSuccess) st = cuda_fail(e, "error-bound clear");
    }
    if (st == SBR_OK && p->n_items > 0) {
        ErrParams P{};
        P.S = s->view();
        P.freqs = p->d_freqs;
        P.dfield = d_dfield;
        P.segs = p->d_segs;
        P.seg_item_base = p->d_seg_base;
        P.n_segs = (int32_t)p->n_segs;
        P.jobs = p->d_jobs;
        P.n_items = p->n_items;
        P.queue = d_queue;
        P.acc = d_acc;
        const double dx = s->aabb_hi[0] - s->aabb_lo[0], dy = s->aabb_hi[1] - s->aabb_lo[1],
                     dz = s->aabb_hi[2] - s->aabb_lo[2];
        P.diag = float(std::sqrt(dx * dx + dy * dy + dz * dz));
        P.err = p->d_err;
        P.cancel = p->d_cancel;
        int occ = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_errbound, kCtaThreads, 0);
        if (e != cudaSuccess) st = cuda_fail(e, "occupancy");
        if (st == SBR_OK) {
            const long long grid = std::min<long long>((long long)std::max(occ, 1) * p->num_sms, (p->n_items + 3) / 4);
            k_errbound<<<(unsigned)std::max(grid, 1LL), kCtaThreads, 0, p->stream>>>(P);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
            if (e != cudaSuccess) st = cuda_fail(e, "error-bound pass");
        }
        if (st == SBR_OK) {
            uint32_t de = 0;
            e = cudaMemcpy(&de, p->d_err, sizeof(de), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) st = cuda_fail(e, "error word");
            else if (de) {
                clear_device_word(p->d_err);
                st = (de & DEV_ERR_CANCEL) ? fail(SBR_ERR_CANCELLED, "run cancelled")
                     : (de & DEV_ERR_BUDGET) ? fail(SBR_ERR_TIMEOUT, "traversal iteration budget exceeded")
                                             : fail(SBR_ERR_STACK, "traversal stack overflow");
            }
        }
    }
    if (st == SBR_OK) {
        e = cudaMemcpy(acc.data(), d_acc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(dfield.data(), d_dfield, dfield.size() * sizeof(double),
                                             cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cuda_fail(e, "error-bound copy");
    }
    if (st == SBR_OK) {
        for (int64_t g = 0; g < p->n_segs; ++g) {
            const Segment& G = p->segs[(size_t)g];
            const JobConst& J = p->jobs[(size_t)G.job];
            const int64_t items = p->seg_base[(size_t)g + 1] - p->seg_base[(size_t)g];
            for (int k = 0; k < J.n_freqs; ++k) {
                const FreqConst& F = p->freqs[(size_t)(J.freq_base + k)];
                const int64_t smp = G.sample_base + k;
                const double* A = acc.data() + 8 * g;
                const double a = std::hypot(field[2 * smp], field[2 * smp + 1]);
                const double shared = a * ((A[0] > 0.0 ? 2.0 * F.k * A[1] / A[0] : 0.0) + kPhaseEps);
                const double E = std::hypot(dfield[2 * smp], dfield[2 * smp + 1]) + shared +
                                 kLambda * F.scale * (2.0 * F.k * std::sqrt(A[3]) + std::sqrt(A[4])) +
                                 double(items + 1) * F.quantum + kLambda * F.scale * double(kU) * std::sqrt(A[2]);
                if (err_field) err_field[smp] = E;
                if (err_db) {
                    const double db = 10.0 * std::log10(std::max(4.0 * M_PI * a * a, 1e-10));
                    const double hi = 10.0 * std::log10(std::max(4.0 * M_PI * (a + E) * (a + E), 1e-10));
                    const double lo_a = std::max(a - E, 0.0);
                    const double lo = 10.0 * std::log10(std::max(4.0 * M_PI * lo_a * lo_a, 1e-10));
                    err_db[smp] = std::max(hi - db, db - lo);
                }
            }
        }
    }
    cudaFree(d_acc);
    cudaFree(d_dfield);
    cudaFree(d_queue);
    sbr_plan_destroy(p);
    return st;
}
