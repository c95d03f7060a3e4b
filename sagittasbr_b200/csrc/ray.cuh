// ray.cuh -- per-ray state of the SBR bounce loop on sm_100a, shared by the sweep
// kernel (trace.cu) and the adjoint kernel (adjoint.cu): primary ray origins, one
// closest-hit query with PEC reflection and nudge, and the scalar exit-ray
// quantities of the PO term (src/cuda/rtKernels.cu:105-158,
// src/cuda/poKernels.cu:81-109).
#pragma once

#include "trace.cuh"

namespace sbr {

// State of one ray between closest-hit queries.
struct RayF {
    F3 o, d, nl, dl;  // nl, dl: last hit normal and incoming direction (records, polarisation)
    float cosl;       // n.(-d_in) at the last hit (the PO gate and obliquity)
    double L;       // FP64 path (mixed)
    float dist32;   // FP32 path (reference FP32 arithmetic)
    int count;
    int zidx;       // entry of this ray in the first-hit buffer
};
struct RayD {
    D3 o, d, nl, dl;
    double cosl;
    double L;
    int count;
};

// What the PO epilogue needs from a finished ray.
struct RayOut {
    float amp;     // 2 cos(theta) R^n, 0 when the ray adds nothing
    float dist32;
    double L;
    float cosT, Rn;
    double cosD, RnD;
    double pa[2];  // SBR_POL_HHVV: co-polarised amplitudes (HH, VV)
    double Lp;     // SBR_POL_HHVV: path launch plane -> exit point -> launch plane
    float Lh, Ll;  // MIXED: the phase path (L, or Lp / 2 for SBR_POL_HHVV) as an FP32 pair
};

// Polarisation state of SBR_POL_HHVV plans: the HH and VV incident fields as they
// arrive at the ray's latest hit (unit vectors; PEC reflection keeps them real).
struct PolF {
    F3 h, v;
};
struct PolD {
    D3 h, v;
};

// PEC boundary condition: the reflected field is 2 (n.E) n - E (tangential part
// reversed, normal part kept).
__device__ __forceinline__ F3 pec_reflect(F3 e, F3 n) { return fma3(2.0f * dot(n, e), n, f3(-e.x, -e.y, -e.z)); }
__device__ __forceinline__ D3 pec_reflect(D3 e, D3 n) {
    const double s = 2.0 * dot(n, e);
    return D3{s * n.x - e.x, s * n.y - e.y, s * n.z - e.z};
}

// Specular reflection of direction d at unit normal n, and the hit point p moved
// off the surface along n: the bounce step of every FP32 / mixed and FP64 ray.
__device__ __forceinline__ F3 reflect_dir(F3 d, F3 n) { return unit(fma3(-(2.0f * dot(d, n)), n, d)); }
__device__ __forceinline__ D3 reflect_dir(D3 d, D3 n) { return unit(d - (2.0 * dot(d, n)) * n); }
__device__ __forceinline__ F3 nudge(F3 p, F3 n) { return fma3(1.0e-4f, n, p); }
__device__ __forceinline__ D3 nudge(D3 p, D3 n) { return p + 1.0e-4 * n; }

// Co-polarised exit amplitude: 2 R^n e.(n x (d_in x E_in)), the direction of the PO
// surface current n x H_in on the last surface projected on the receive
// polarisation e, with the scalar term's ray-tube weighting.  For a single bounce
// (E_in = e, d_in = -s) it equals the scalar amplitude 2 cos(theta) R^n.
template <class V, class R>
__device__ __forceinline__ R pol_amp(V e, V n, V d, V E, R twoRn) {
    return twoRn * dot(e, cross(n, cross(d, E)));
}

// x as an unevaluated FP32 pair hi + lo (|x - hi - lo| <= 2^-48 |x|).
__device__ __forceinline__ void split_f32(double x, float& hi, float& lo) {
    hi = float(x);
    lo = float(x - double(hi));
}

// ------------------------------------------------------------ FP32 / mixed
// Origin of the primary ray of pixel (i, j) (src/cuda/rtKernels.cu:120-123); the
// trace and the first-hit raster both use this, so they test identical rays.
template <int PREC>
__device__ __forceinline__ F3 primary_origin(const Segment& G, const JobConst& J, int i, int j) {
    if (PREC == SBR_PREC_FP32) {
        const float u = __fdiv_rn(float(i) + 0.5f, float(J.nx));
        const float v = __fdiv_rn(float(j) + 0.5f, float(J.ny));
        return fma3(v, f3(G.vf[0], G.vf[1], G.vf[2]),
                    fma3(u, f3(G.uf[0], G.uf[1], G.uf[2]), f3(G.llcf[0], G.llcf[1], G.llcf[2])));
    } else {
        const double u = (double(i) + 0.5) * J.inv_nx;
        const double v = (double(j) + 0.5) * J.inv_ny;
        const D3 o = fma3(v, D3{G.v[0], G.v[1], G.v[2]}, fma3(u, D3{G.u[0], G.u[1], G.u[2]}, D3{G.llc[0], G.llc[1], G.llc[2]}));
        return f3(float(o.x), float(o.y), float(o.z));
    }
}

// First-hit buffer entry of ray (i, j): tile-major, the lane of the 4x8 block last.
__device__ __forceinline__ int zindex(const Segment& G, int i, int j) {
    const int bi = i - G.i0, bj = j - G.j0;
    return (int)(G.zbase + 32 * (int64_t)((bj >> 3) * G.blocks_x + (bi >> 2)) + ((bj & 7) << 2) + (bi & 3));
}

template <int PREC>
__device__ __forceinline__ void start_f(RayF& r, const Segment& G, const JobConst& J, int i, int j) {
    r.o = primary_origin<PREC>(G, J, i, j);
    r.L = PREC == SBR_PREC_FP32 ? 0.0 : G.shift;
    r.zidx = zindex(G, i, j);
    r.d = f3(G.rdf[0], G.rdf[1], G.rdf[2]);
    r.nl = f3(0, 0, 0);
    r.dl = f3(0, 0, 0);
    r.cosl = 0.0f;
    r.dist32 = 0.0f;
    r.count = 0;
}

// First-hit buffer entries: (t bits << 32) | slot for a hit, kZMiss for none, and
// kZWalk where the ray's first query walks the tree (its tile's triangle list was
// too long to test); the high word of a hit is a finite positive float.
constexpr unsigned long long kZMiss = ~0ull;
constexpr unsigned long long kZWalk = 0xfffffffe00000000ull;

// One closest-hit query, then reflect and nudge; true when the ray is finished.
// The first query is read from the first-hit buffer when there is one.
// SPEC: the speculative closest-hit walk, entered by all lanes of `mask` together.
template <int PREC, bool REC, bool POL, bool W8 = false, bool SPEC = false>
__device__ __forceinline__ bool step_f(RayF& r, PolF& e, const SceneView& S, int maxB, uint32_t& err,
                                       sbr_ray_record* rec, unsigned long long* zbuf, unsigned mask = 0u) {
    float tB = 1e20f;
    int slot;
    const unsigned long long key = (zbuf != nullptr && r.count == 0) ? zbuf[r.zidx] : kZWalk;
    if (key == kZMiss) return true;
    if (key != kZWalk) {
        tB = __uint_as_float((unsigned)(key >> 32));
        slot = (int)(unsigned)key;
    } else if constexpr (SPEC) {
        static_assert(PREC == SBR_PREC_MIXED && !REC && !POL && !W8, "the speculative walk is the mixed scalar sweep's");
        slot = closest_speculative(S, r.o, r.d, 1.0e-3f, tB, err, mask);
    } else if constexpr (W8) {
        static_assert(PREC == SBR_PREC_MIXED && !REC && !POL, "the 8-wide walk is the mixed scalar sweep's");
        slot = Walker8::closest(S, r.o, r.d, 1.0e-3f, tB, err);
    } else {
        slot = Walker<false>::closest<PREC == SBR_PREC_MIXED, !REC && !POL>(S, r.o, r.d, 1.0e-3f, tB, err);
    }
    if (slot < 0) return true;
    const GTri* T = S.tris + slot;
    const F3 n = f3(__ldg(&T->v0.w), __ldg(&T->v1.w), __ldg(&T->v2.w));
    if constexpr (POL) {
        if (r.count > 0) {  // the field left the previous hit reflected there
            e.h = pec_reflect(e.h, r.nl);
            e.v = pec_reflect(e.v, r.nl);
        }
    }
    r.cosl = dot(n, f3(-r.d.x, -r.d.y, -r.d.z));
    r.nl = n;
    r.dl = r.d;
    ++r.count;
    if (PREC == SBR_PREC_FP32) r.dist32 += tB;
    else r.L += double(tB);
    if (REC && r.count <= SBR_MAX_REC) rec->tri[r.count - 1] = __ldg(S.tri_id + slot);
    const F3 p = fma3(tB, r.d, r.o);
    r.d = reflect_dir(r.d, n);
    r.o = nudge(p, n);
    return r.count >= maxB;
}

template <int PREC>
__device__ __forceinline__ RayOut finish_f(const RayF& r, const JobConst& J) {
    RayOut o;
    float Rn = 1.0f;
    for (int b = 0; b < r.count; ++b) Rn *= J.reflf;
    const float c = r.cosl;
    o.cosT = c;
    o.Rn = Rn;
    o.cosD = c;
    o.RnD = Rn;
    o.dist32 = r.dist32;
    o.L = (PREC == SBR_PREC_FP32) ? double(r.dist32) : r.L;
    o.amp = (r.count > 0 && c > 0.0f) ? 2.0f * c * Rn : 0.0f;
    split_f32(o.L, o.Lh, o.Ll);
    return o;
}

// --------------------------------------------------------------------- FP64
__device__ __forceinline__ void start_d(RayD& r, const Segment& G, const JobConst& J, int i, int j) {
    const double u = (double(i) + 0.5) / double(J.nx);
    const double v = (double(j) + 0.5) / double(J.ny);
    r.o = D3{G.llc[0] + u * G.u[0] + v * G.v[0], G.llc[1] + u * G.u[1] + v * G.v[1],
             G.llc[2] + u * G.u[2] + v * G.v[2]};
    r.d = D3{-G.dir[0], -G.dir[1], -G.dir[2]};
    r.nl = D3{0, 0, 0};
    r.dl = D3{0, 0, 0};
    r.cosl = 0.0;
    r.L = G.shift;
    r.count = 0;
}

template <bool REC, bool POL>
__device__ __forceinline__ bool step_d(RayD& r, PolD& e, const SceneView& S, int maxB, uint32_t& err,
                                       sbr_ray_record* rec) {
    double tB = 1e20;
    const int slot = Walker<true>::closest(S, r.o, r.d, 1.0e-3, tB, err);
    if (slot < 0) return true;
    const GTri64& T = S.tris64[slot];
    // the hit normal unit(e1 x e2) formed here, as the reference forms it on the
    // device for every hit (src/cuda/rtKernels.cu:42), not the host's copy
    const D3 n = unit(cross(D3{T.e1[0], T.e1[1], T.e1[2]}, D3{T.e2[0], T.e2[1], T.e2[2]}));
    if constexpr (POL) {
        if (r.count > 0) {
            e.h = pec_reflect(e.h, r.nl);
            e.v = pec_reflect(e.v, r.nl);
        }
    }
    r.cosl = dot(n, D3{-r.d.x, -r.d.y, -r.d.z});
    r.nl = n;
    r.dl = r.d;
    ++r.count;
    r.L += tB;
    if (REC && r.count <= SBR_MAX_REC) rec->tri[r.count - 1] = __ldg(S.tri_id + slot);
    const D3 p = r.o + tB * r.d;
    r.d = reflect_dir(r.d, n);
    r.o = nudge(p, n);
    return r.count >= maxB;
}

__device__ __forceinline__ RayOut finish_d(const RayD& r, const JobConst& J) {
    RayOut o;
    double Rn = 1.0;
    for (int b = 0; b < r.count; ++b) Rn *= J.refl;
    const double c = r.cosl;
    o.cosT = float(c);
    o.Rn = float(Rn);
    o.cosD = c;
    o.RnD = Rn;
    o.L = r.L;
    o.dist32 = float(r.L);
    o.amp = (r.count > 0 && c > 0.0) ? float(2.0 * c * Rn) : 0.0f;
    split_f32(o.L, o.Lh, o.Ll);
    return o;
}

// ------------------------------------------------------------ PO term
// The MIXED phase, (k / pi) L turns, is formed and reduced in FP32 arithmetic on
// unevaluated pairs (hi + lo; Dekker, Numer. Math. 18, 1971): the product of the
// leading parts is split exactly into p + e by one FMA, the cross products are
// added to e, and the whole turns are taken from p alone, p - rint(p) being exact
// in FP32.  The remainder r = (p - rint(p)) + e lies within 2^-25 + 2^-45 |x|
// turns of the exact one (x = k L / pi; |x| < 2^17, a 1 km path at 18 GHz, gives
// 3.4e-8 turns) and |r| <= 1/2 + 2^-24 |x|.  No FP64 operation and no
// conversion per (ray, frequency): only the sine and cosine use the special
// function unit.
__device__ __forceinline__ float turns_frac(float th, float tl, float Lh, float Ll) {
    const float p = th * Lh;
    float e = fmaf(th, Lh, -p);
    e = fmaf(th, Ll, e);
    e = fmaf(tl, Lh, e);
    return (p - rintf(p)) + e;
}
// sin and cos of the MIXED phase of path (Lh + Ll) at frequency F.
__device__ __forceinline__ void sincos_mixed(const FreqConst& F, float Lh, float Ll, float& s, float& c) {
    __sincosf(6.28318530717958647692f * turns_frac(F.turns_hi, F.turns_lo, Lh, Ll), &s, &c);
}

// PO term of one ray at one frequency, added to (re, im).
//  FP32: the reference FP32 arithmetic (phase fmodf in FP32).
//  MIXED: phase 2 k L = 2 pi (k / pi) L reduced in turns (sincos_mixed); the
//         term is summed without the factor k A / (4 pi), which the item fold
//         applies once per channel.
//  FP64: the reference USE_DOUBLE arithmetic.
__device__ __forceinline__ void po_term(int prec, const FreqConst& F, const RayOut& r, double& re, double& im) {
    if (prec == SBR_PREC_FP32) {
        const float twoPi = 6.28318548202514648438f;
        float phase = (2.0f * F.kf) * r.dist32;
        phase = fmodf(phase, twoPi);
        const float mag = (F.scalef * 2.0f) * r.cosT * r.Rn;
        float s, c;
        sincosf(phase, &s, &c);
        re += double(-mag * s);
        im += double(mag * c);
    } else if (prec == SBR_PREC_MIXED) {
        float s, c;
        sincos_mixed(F, r.Lh, r.Ll, s, c);
        const double a = double(r.amp);
        re -= a * double(s);
        im += a * double(c);
    } else {
        const double twoPi = 2.0 * 3.14159265358979323846;
        const double phase = fmod((2.0 * F.k) * r.L, twoPi);
        const double mag = (F.scale * 2.0) * r.cosD * r.RnD;
        double s, c;
        sincos(phase, &s, &c);
        re += -mag * s;
        im += mag * c;
    }
}

}  // namespace sbr
