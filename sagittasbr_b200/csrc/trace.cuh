// trace.cuh -- device building blocks of the SBR path for sm_100a:
// closest-hit traversal of the 4-wide BVH, the bounce loop with PEC reflection and
// the reference's scalar PO exit-ray term.
//
// Semantics follow the reference per-ray routine:
//   ray origin at pixel centres ................ src/cuda/rtKernels.cu:118-123
//   closest hit with tMin = 1e-3, tMax = 1e20 ... src/cuda/rtKernels.cu:136
//   Moller-Trumbore, two-sided, |det| < 1e-6 .... src/cuda/rtKernels.cu:10-44
//   normal unit(e1 x e2) ........................ src/cuda/rtKernels.cu:42
//   reflect d - 2 (d.n) n, nudge p + 1e-4 n ..... src/cuda/rtKernels.cu:146-152
//   PO: R^n, cos = n.(-d_last) > 0, phase 2 k L, mag = k A / (4 pi) * 2 cos R^n,
//       term (-mag sin, mag cos) ............... src/cuda/poKernels.cu:81-109
// The traversal order differs from the reference (nearest child first, entries
// beyond the current closest hit are skipped, 4-wide nodes); it returns the same
// closest hit except for exact ties between triangles (shared edges), where the
// reference keeps the last triangle tested.
#pragma once

#include "common.hpp"

namespace sbr {

// ------------------------------------------------------------ small vectors
struct F3 {
    float x, y, z;
};
struct D3 {
    double x, y, z;
};
// The FP32 / mixed ray arithmetic is written with explicitly rounded operations
// (__fadd_rn, __fmul_rn, __fmaf_rn, ...: each rounded once as written, never
// contracted or split by the compiler), so every kernel that starts, reflects or
// tests a ray -- the sweep in each of its epilogue layouts, the record and ray-list
// traces, the first-hit raster, the error bound's re-trace -- computes it bit for
// bit the same way.  Products that are summed are fused (dot and cross products,
// a s + b).
__device__ __forceinline__ F3 f3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) {
    return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)};
}
__device__ __forceinline__ F3 operator-(F3 a, F3 b) {
    return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
__device__ __forceinline__ F3 operator*(float s, F3 a) { return {__fmul_rn(s, a.x), __fmul_rn(s, a.y), __fmul_rn(s, a.z)}; }
// s a + b, one rounding per component
__device__ __forceinline__ F3 fma3(float s, F3 a, F3 b) {
    return {__fmaf_rn(s, a.x, b.x), __fmaf_rn(s, a.y, b.y), __fmaf_rn(s, a.z, b.z)};
}
__device__ __forceinline__ float dot(F3 a, F3 b) { return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x))); }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
    return {__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)), __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
            __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x))};
}
// Normalisation with the hardware reciprocal square root (a few ulp, like the
// reference's --use_fast_math FP32 build).
__device__ __forceinline__ F3 unit(F3 a) {
    const float r = rsqrtf(dot(a, a));
    return {__fmul_rn(a.x, r), __fmul_rn(a.y, r), __fmul_rn(a.z, r)};
}
// FP64 vectors keep the compiler's plain evaluation, as the reference's USE_DOUBLE
// build is compiled, so the FP64 mode reproduces that build's arithmetic; fma3 is
// the explicitly fused form for the mixed-precision ray origins.
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ D3 fma3(double s, D3 a, D3 b) {
    return {__fma_rn(s, a.x, b.x), __fma_rn(s, a.y, b.y), __fma_rn(s, a.z, b.z)};
}
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// written as the reference's vec3 cross (include/RT/vec3.h:115-119), y negated, so
// the compiler fuses the same products
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, -(a.x * b.z - a.z * b.x), a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 unit(D3 a) {
    double l = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return {a.x / l, a.y / l, a.z / l};
}

// Three-input min / max (sm_100 PTX); like fminf/fmaxf they return the other
// operand when one is NaN.
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Reciprocal direction for the slab tests.  Components below 1e-20 in magnitude
// are clamped (keeps the slab arithmetic finite, no 0 * inf); the approximate
// reciprocal's relative error (< 2^-22) is covered by the slab slack below.
__device__ __forceinline__ float slab_inv(float d) {
    float c = fabsf(d) > 1e-20f ? d : copysignf(1e-20f, d);
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(c));
    return r;
}
__device__ __forceinline__ double slab_inv(double d) { return 1.0 / (fabs(d) > 1e-200 ? d : copysign(1e-200, d)); }

// Entry distance of a box, +inf when missed.  Boxes are conservative; the exit is
// widened by a relative 2^-20 so neither the FMA form nor the approximate
// reciprocal ever rejects a box the ray touches (boxes only prune, the triangle
// test decides every hit).
constexpr float kSlabSlack = 1.00000095367431640625f;  // 1 + 2^-20
__device__ __forceinline__ float slab_f(float lx, float hx, float ly, float hy, float lz, float hz, F3 inv, F3 oi,
                                        float tMin, float tMax) {
    float x0 = fmaf(lx, inv.x, -oi.x), x1 = fmaf(hx, inv.x, -oi.x);
    float y0 = fmaf(ly, inv.y, -oi.y), y1 = fmaf(hy, inv.y, -oi.y);
    float z0 = fmaf(lz, inv.z, -oi.z), z1 = fmaf(hz, inv.z, -oi.z);
    float tn = max3f(fminf(x0, x1), fminf(y0, y1), fmaxf(fminf(z0, z1), tMin));
    float tf = min3f(fmaxf(x0, x1), fmaxf(y0, y1), fminf(fmaxf(z0, z1), tMax));
    return tn <= tf * kSlabSlack ? tn : __int_as_float(0x7f800000);
}
// The same entry distance with the planes already ordered by the ray's direction
// signs (near plane first on every axis): fma is monotone in the plane coordinate,
// so this equals slab_f bit for bit without the six per-axis min / max.
__device__ __forceinline__ float slab_nf(float nx, float fx, float ny, float fy, float nz, float fz, F3 inv, F3 oi,
                                         float tMin, float tMax) {
    const float tn = max3f(fmaf(nx, inv.x, -oi.x), fmaf(ny, inv.y, -oi.y), fmaxf(fmaf(nz, inv.z, -oi.z), tMin));
    const float tf = min3f(fmaf(fx, inv.x, -oi.x), fmaf(fy, inv.y, -oi.y), fminf(fmaf(fz, inv.z, -oi.z), tMax));
    return tn <= tf * kSlabSlack ? tn : __int_as_float(0x7f800000);
}
// slab_nf as an entry distance and an acceptance flag, without materialising +inf
// for rejected boxes: `hit` is tn <= tf (1 + 2^-20) with tf already clamped to tMax,
// so an accepted entry lies at most 2^-20 relative beyond tMax (boxes only prune).
__device__ __forceinline__ float slab_nh(float nx, float fx, float ny, float fy, float nz, float fz, F3 inv, F3 oi,
                                         float tMin, float tMax, bool& hit) {
    const float tn = max3f(fmaf(nx, inv.x, -oi.x), fmaf(ny, inv.y, -oi.y), fmaxf(fmaf(nz, inv.z, -oi.z), tMin));
    const float tf = min3f(fmaf(fx, inv.x, -oi.x), fmaf(fy, inv.y, -oi.y), fminf(fmaf(fz, inv.z, -oi.z), tMax));
    hit = tn <= tf * kSlabSlack;
    return tn;
}
// Two-wide FP32 (sm_100 `fma.rn.f32x2`): both halves rounded exactly as fmaf, so
// a pair of slab planes costs one instruction and equals the scalar form bit for bit.
__device__ __forceinline__ unsigned long long pack2(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b,
                                                   unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
// Ray constants of slab4_nh: every axis' reciprocal direction and -o * inv, each
// duplicated into both halves of a pair.
struct Slab2 {
    unsigned long long ix, iy, iz, ox, oy, oz;
};
__device__ __forceinline__ Slab2 slab2(F3 inv, F3 oi) {
    return {pack2(inv.x, inv.x), pack2(inv.y, inv.y), pack2(inv.z, inv.z),
            pack2(-oi.x, -oi.x), pack2(-oi.y, -oi.y), pack2(-oi.z, -oi.z)};
}
// slab_nh for the four children of a node at once (planes already ordered by the
// ray's direction signs): the 24 plane distances as 12 two-wide FMAs, children
// (0, 1) and (2, 3) paired.  Same entry distances and flags as four slab_nh calls.
__device__ __forceinline__ void slab4_nh(const float4& nx, const float4& fx, const float4& ny, const float4& fy,
                                         const float4& nz, const float4& fz, const Slab2& R, float tMin, float tMax,
                                         float (&t)[4], bool (&h)[4]) {
    float xn[4], xf[4], yn[4], yf[4], zn[4], zf[4];
    unpack2(fma2(pack2(nx.x, nx.y), R.ix, R.ox), xn[0], xn[1]);
    unpack2(fma2(pack2(nx.z, nx.w), R.ix, R.ox), xn[2], xn[3]);
    unpack2(fma2(pack2(fx.x, fx.y), R.ix, R.ox), xf[0], xf[1]);
    unpack2(fma2(pack2(fx.z, fx.w), R.ix, R.ox), xf[2], xf[3]);
    unpack2(fma2(pack2(ny.x, ny.y), R.iy, R.oy), yn[0], yn[1]);
    unpack2(fma2(pack2(ny.z, ny.w), R.iy, R.oy), yn[2], yn[3]);
    unpack2(fma2(pack2(fy.x, fy.y), R.iy, R.oy), yf[0], yf[1]);
    unpack2(fma2(pack2(fy.z, fy.w), R.iy, R.oy), yf[2], yf[3]);
    unpack2(fma2(pack2(nz.x, nz.y), R.iz, R.oz), zn[0], zn[1]);
    unpack2(fma2(pack2(nz.z, nz.w), R.iz, R.oz), zn[2], zn[3]);
    unpack2(fma2(pack2(fz.x, fz.y), R.iz, R.oz), zf[0], zf[1]);
    unpack2(fma2(pack2(fz.z, fz.w), R.iz, R.oz), zf[2], zf[3]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float tn = max3f(xn[k], yn[k], fmaxf(zn[k], tMin));
        const float tf = min3f(xf[k], yf[k], fminf(zf[k], tMax));
        h[k] = tn <= tf * kSlabSlack;
        t[k] = tn;
    }
}
__device__ __forceinline__ double slab_d(double lx, double hx, double ly, double hy, double lz, double hz, D3 o,
                                         D3 inv, double tMin, double tMax) {
    double x0 = (lx - o.x) * inv.x, x1 = (hx - o.x) * inv.x;
    double y0 = (ly - o.y) * inv.y, y1 = (hy - o.y) * inv.y;
    double z0 = (lz - o.z) * inv.z, z1 = (hz - o.z) * inv.z;
    double tn = fmax(fmax(fmin(x0, x1), fmin(y0, y1)), fmax(fmin(z0, z1), tMin));
    double tf = fmin(fmin(fmax(x0, x1), fmax(y0, y1)), fmin(fmax(z0, z1), tMax));
    return tn <= tf * (1.0 + 1e-12) ? tn : __longlong_as_double(0x7ff0000000000000LL);
}

// Moller-Trumbore in the reference's operation order.
__device__ __forceinline__ bool mt_f(const GTri& T, F3 o, F3 d, float tMin, float tMax, float& t) {
    const F3 v0 = f3(T.v0.x, T.v0.y, T.v0.z);
    F3 e1 = f3(T.v1.x, T.v1.y, T.v1.z) - v0, e2 = f3(T.v2.x, T.v2.y, T.v2.z) - v0;
    F3 pv = cross(d, e2);
    float det = dot(e1, pv);
    if (fabsf(det) < 1.0e-6f) return false;
    float inv = __frcp_rn(det);
    F3 tv = o - v0;
    float u = dot(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    F3 qv = cross(tv, e1);
    float v = dot(d, qv) * inv;
    if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return false;
    float tt = dot(e2, qv) * inv;
    if (tt < tMin || tt > tMax) return false;
    t = tt;
    return true;
}

// Watertight ray / triangle test (Woop, Benthin and Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2(1), 2013), two-sided, FP32.  The vertices are moved to the
// ray origin and sheared so the ray runs along the axis kz of its largest direction
// component; the three 2-D edge functions U, V, W of the sheared triangle are then
// formed without FMA contraction, so a shared edge evaluates to exactly opposite
// values in its two triangles and no ray passes between them (a zero falls back to
// FP64, where the products are exact).  Accepted as by the reference's
// Moller-Trumbore otherwise: |det| < 1e-6 rejected (|det_MT| = |U + V + W| |d_kz|),
// t in [tMin, tMax]; t = T / det with the approximate reciprocal (2 ulp).
struct WtRay {
    int kz;         // dominant axis of d; kx = kz + 1, ky = kz + 2 (mod 3)
    float sx, sy;   // d[kx] / d[kz], d[ky] / d[kz] (to 2 ulp)
    float sz;       // 1 / d[kz] (to 2 ulp)
    float adz;      // |d[kz]|
};
__device__ __forceinline__ WtRay wt_ray(F3 d) {
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    WtRay w;
    w.kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    const float dz = w.kz == 0 ? d.x : w.kz == 1 ? d.y : d.z;
    const float dx = w.kz == 0 ? d.y : w.kz == 1 ? d.z : d.x;
    const float dy = w.kz == 0 ? d.z : w.kz == 1 ? d.x : d.y;
    // any per-ray constants keep the test watertight (each vertex is transformed the
    // same way for every triangle); the approximate reciprocal is enough
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(w.sz) : "f"(dz));
    w.sx = __fmul_rn(dx, w.sz);
    w.sy = __fmul_rn(dy, w.sz);
    w.adz = fabsf(dz);
    return w;
}
template <int K>
__device__ __forceinline__ float axis(const float4& v) {
    return K == 0 ? v.x : K == 1 ? v.y : v.z;
}
template <int K>
__device__ __forceinline__ float axis(F3 v) {
    return K == 0 ? v.x : K == 1 ? v.y : v.z;
}
template <int KZ>
__device__ __forceinline__ bool wt_tri(const GTri& T, F3 o, const WtRay& w, float tMin, float tMax, float& t) {
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
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (!(fabsf(det) * w.adz >= 1.0e-6f)) return false;
    const float T3 = __fmaf_rn(U, az, __fmaf_rn(V, bz, __fmul_rn(W, cz)));
    float rdet;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rdet) : "f"(det));
    const float tt = __fmul_rn(__fmul_rn(T3, w.sz), rdet);
    if (!(tt >= tMin && tt <= tMax)) return false;
    t = tt;
    return true;
}
// A hit at tt (<= tBest) of triangle `slot` replaces the closest one so far when it
// is nearer, or none is kept yet (best = -1), or it is as near and comes later in
// the tie order: the rank of the triangle in the reference's walk (tie[slot]; the
// reference keeps the last of equally near triangles), or, where the scene stores
// no ranks (no coincident faces of opposite winding), the slot order reversed.  The
// closest hit does not depend on the order triangles are tested in, so the walk and
// the first-hit raster keep the same triangle on exact ties.
__device__ __forceinline__ bool tie_later(int slot, int best, const int32_t* __restrict__ tie) {
    return tie ? __ldg(tie + slot) > __ldg(tie + best) : slot < best;
}
__device__ __forceinline__ bool replaces(float tt, int slot, float tBest, int best, const int32_t* tie) {
    return tt < tBest || best < 0 || tie_later(slot, best, tie);
}
__device__ __forceinline__ bool replaces(double tt, int slot, double tBest, int best, const int32_t* tie) {
    return tt < tBest || best < 0 || tie_later(slot, best, tie);
}
// A leaf's triangles with the axis order fixed at compile time: the switch on kz
// sits outside the loop, so a warp whose rays share a dominant axis runs one variant.
template <int KZ>
__device__ __forceinline__ void leaf_wt(const GTri* __restrict__ tris, const int32_t* tie, int first, int cnt, F3 o,
                                        const WtRay& w, float tMin, float& tBest, int& best) {
    for (int k = 0; k < cnt; ++k) {
        float tt;
        if (wt_tri<KZ>(tris[first + k], o, w, tMin, tBest, tt) && replaces(tt, first + k, tBest, best, tie)) {
            tBest = tt;
            best = first + k;
        }
    }
}
__device__ __forceinline__ bool wt_f(const GTri& T, F3 o, const WtRay& w, float tMin, float tMax, float& t) {
    switch (w.kz) {
        case 0: return wt_tri<0>(T, o, w, tMin, tMax, t);
        case 1: return wt_tri<1>(T, o, w, tMin, tMax, t);
        default: return wt_tri<2>(T, o, w, tMin, tMax, t);
    }
}

__device__ __forceinline__ bool mt_d(const GTri64& T, D3 o, D3 d, double tMin, double tMax, double& t) {
    D3 e1{T.e1[0], T.e1[1], T.e1[2]}, e2{T.e2[0], T.e2[1], T.e2[2]};
    D3 pv = cross(d, e2);
    double det = dot(e1, pv);
    if (fabs(det) < 1.0e-6) return false;
    double inv = 1.0 / det;
    D3 tv = o - D3{T.v0[0], T.v0[1], T.v0[2]};
    double u = dot(tv, pv) * inv;
    if (u < 0.0 || u > 1.0) return false;
    D3 qv = cross(tv, e1);
    double v = dot(d, qv) * inv;
    if (v < 0.0 || u + v > 1.0) return false;
    double tt = dot(e2, qv) * inv;
    if (tt < tMin || tt > tMax) return false;
    t = tt;
    return true;
}

__device__ __forceinline__ GNode4 load_node(const GNode4* p) {
    GNode4 n;
    n.lox = __ldg(&p->lox);
    n.hix = __ldg(&p->hix);
    n.loy = __ldg(&p->loy);
    n.hiy = __ldg(&p->hiy);
    n.loz = __ldg(&p->loz);
    n.hiz = __ldg(&p->hiz);
    n.child = __ldg(&p->child);
    return n;
}

// Sorts four (entry distance, child) pairs by distance, nearest first (five
// compare-exchanges, no branches; misses carry +inf and end up last).
template <typename T>
__device__ __forceinline__ void cswap(T& ta, int& ca, T& tb, int& cb) {
    const bool s = tb < ta;
    const T t = s ? tb : ta;
    tb = s ? ta : tb;
    ta = t;
    const int c = s ? cb : ca;
    cb = s ? ca : cb;
    ca = c;
}
template <typename T>
__device__ __forceinline__ void sort4(T (&t)[4], int (&c)[4]) {
    cswap(t[0], c[0], t[1], c[1]);
    cswap(t[2], c[2], t[3], c[3]);
    cswap(t[0], c[0], t[2], c[2]);
    cswap(t[1], c[1], t[3], c[3]);
    cswap(t[1], c[1], t[2], c[2]);
}

constexpr uint32_t kIterBudget = 1u << 22;  // node + leaf steps per query before giving up

// Stack entry: child reference in the low word, entry distance (float bits, or the
// FP64 distance rounded down to float) in the high word.
__device__ __forceinline__ unsigned long long pack_entry(int ref, float t) {
    return ((unsigned long long)__float_as_uint(t) << 32) | (unsigned)ref;
}

// Closest hit along o + t d with t in [tMin, tBest]: returns the leaf slot of the hit
// triangle (or -1) and lowers tBest to its distance.  While-while structure over
// 4-wide nodes: the children a ray's slab test accepts are ordered by entry
// distance, the nearest is entered and the others are pushed (farthest first) with
// their entry distances; leaves are tested, popped entries beyond the current hit
// are skipped.  `err` collects DEV_ERR_* bits.
template <bool kF64>
struct Walker;

// The FP32 walker tests triangles with the watertight test (kWT) or with the
// reference's Moller-Trumbore.  kF2 computes the slab planes two-wide: faster where
// registers are free (the scalar sweep), slower where the six duplicated ray
// constants push other state into local memory (polarised and recording walks).
template <>
struct Walker<false> {
    template <bool kWT, bool kF2 = true>
    __device__ __forceinline__ static int closest(const SceneView& S, F3 o, F3 d, float tMin, float& tBest,
                                                  uint32_t& err) {
        const F3 inv{slab_inv(d.x), slab_inv(d.y), slab_inv(d.z)};
        WtRay wr;
        if constexpr (kWT) wr = wt_ray(d);
        const F3 oi{o.x * inv.x, o.y * inv.y, o.z * inv.z};
        Slab2 R2;
        if constexpr (kF2) R2 = slab2(inv, oi);
        // byte offsets of each axis' near and far planes within a GNode4 (lo planes
        // at 0 / 32 / 64, hi planes 16 bytes after them): the ray's direction signs
        // decide which plane enters a slab, so the loads pick the planes
        const unsigned onx = inv.x < 0.0f ? 16u : 0u, ony = inv.y < 0.0f ? 48u : 32u, onz = inv.z < 0.0f ? 80u : 64u;
        const unsigned ofx = onx ^ 16u, ofy = ony ^ 16u, ofz = onz ^ 16u;
        unsigned long long stack[kStackDepth];
        int sp = 0;
        int ref = 0;
        int best = -1;
        uint32_t iters = 0;
        auto plane = [](const GNode4* p, unsigned off) {
            return __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const char*>(p) + off));
        };
        auto push = [&](int r, float t) {
            if (sp < kStackDepth) stack[sp++] = pack_entry(r, t);
            else err |= DEV_ERR_STACK;
        };
        auto pop = [&]() {
            while (sp > 0) {
                const unsigned long long e = stack[--sp];
                if (__uint_as_float((unsigned)(e >> 32)) <= tBest) { ref = (int)(unsigned)e; return true; }
            }
            return false;
        };
        for (;;) {
            while (ref >= 0) {
                if (++iters > kIterBudget) { err |= DEV_ERR_BUDGET; return -1; }
                const GNode4* np = S.nodes + ref;
                const float4 nx = plane(np, onx), fx = plane(np, ofx), ny = plane(np, ony), fy = plane(np, ofy);
                const float4 nz = plane(np, onz), fz = plane(np, ofz);
                const int4 ch = __ldg(&np->child);
                float t[4];
                bool hh[4];
                if constexpr (kF2) {
                    slab4_nh(nx, fx, ny, fy, nz, fz, R2, tMin, tBest, t, hh);
                } else {
                    t[0] = slab_nh(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, inv, oi, tMin, tBest, hh[0]);
                    t[1] = slab_nh(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, inv, oi, tMin, tBest, hh[1]);
                    t[2] = slab_nh(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, inv, oi, tMin, tBest, hh[2]);
                    t[3] = slab_nh(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, inv, oi, tMin, tBest, hh[3]);
                }
                const bool h0 = hh[0], h1 = hh[1], h2 = hh[2], h3 = hh[3];
                int c[4] = {ch.x, ch.y, ch.z, ch.w};
                // most visits accept exactly one child (no ordering needed); two or
                // more are sorted (rejected children last) and all but the nearest
                // pushed, farthest first
                const int nh = int(h0) + int(h1) + int(h2) + int(h3);
                if (nh == 1) {
                    ref = h0 ? c[0] : h1 ? c[1] : h2 ? c[2] : c[3];
                } else if (nh == 2) {
                    // the first and the last accepted child: enter the nearer, push the other
                    const float ta = h0 ? t[0] : h1 ? t[1] : t[2];
                    const int ca = h0 ? c[0] : h1 ? c[1] : c[2];
                    const float tb = h3 ? t[3] : h2 ? t[2] : t[1];
                    const int cb = h3 ? c[3] : h2 ? c[2] : c[1];
                    const bool sw = tb < ta;
                    push(sw ? ca : cb, sw ? ta : tb);
                    ref = sw ? cb : ca;
                } else if (nh > 2) {
                    const float inf = __int_as_float(0x7f800000);
                    t[0] = h0 ? t[0] : inf;
                    t[1] = h1 ? t[1] : inf;
                    t[2] = h2 ? t[2] : inf;
                    t[3] = h3 ? t[3] : inf;
                    sort4(t, c);
                    if (t[3] <= tBest) push(c[3], t[3]);
                    if (t[2] <= tBest) push(c[2], t[2]);
                    push(c[1], t[1]);
                    ref = c[0];
                } else if (!pop()) {
                    return best;
                }
            }
            do {
                if (++iters > kIterBudget) { err |= DEV_ERR_BUDGET; return -1; }
                const int code = ~ref;
                const int first = code >> 4, cnt = code & 15;
                if constexpr (kWT) {
                    switch (wr.kz) {
                        case 0: leaf_wt<0>(S.tris, S.tie, first, cnt, o, wr, tMin, tBest, best); break;
                        case 1: leaf_wt<1>(S.tris, S.tie, first, cnt, o, wr, tMin, tBest, best); break;
                        default: leaf_wt<2>(S.tris, S.tie, first, cnt, o, wr, tMin, tBest, best); break;
                    }
                } else {
                    for (int k = 0; k < cnt; ++k) {
                        float tt;
                        if (mt_f(S.tris[first + k], o, d, tMin, tBest, tt) && replaces(tt, first + k, tBest, best, S.tie)) {
                            tBest = tt;
                            best = first + k;
                        }
                    }
                }
                if (!pop()) return best;
            } while (ref < 0);
        }
    }
};

// Closest hit over the opt-in 8-wide tree (SceneView::nodes8), mixed precision:
// the watertight triangle test and the two-wide slab planes of the 4-wide walker,
// on both halves of a node.  One accepted child is entered directly; two or more
// are ordered by entry distance (each half sorted, then an odd-even merge: 19
// compare-exchanges), the nearest entered and the rest pushed farthest first.
struct Walker8 {
    __device__ __forceinline__ static int closest(const SceneView& S, F3 o, F3 d, float tMin, float& tBest,
                                                  uint32_t& err) {
        const F3 inv{slab_inv(d.x), slab_inv(d.y), slab_inv(d.z)};
        const WtRay wr = wt_ray(d);
        const F3 oi{o.x * inv.x, o.y * inv.y, o.z * inv.z};
        const Slab2 R2 = slab2(inv, oi);
        const unsigned onx = inv.x < 0.0f ? 16u : 0u, ony = inv.y < 0.0f ? 48u : 32u, onz = inv.z < 0.0f ? 80u : 64u;
        const unsigned ofx = onx ^ 16u, ofy = ony ^ 16u, ofz = onz ^ 16u;
        unsigned long long stack[kStackDepth];
        int sp = 0;
        int ref = 0;
        int best = -1;
        uint32_t iters = 0;
        auto plane = [](const GNode4* p, unsigned off) {
            return __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const char*>(p) + off));
        };
        auto push = [&](int r, float t) {
            if (sp < kStackDepth) stack[sp++] = pack_entry(r, t);
            else err |= DEV_ERR_STACK;
        };
        auto pop = [&]() {
            while (sp > 0) {
                const unsigned long long e = stack[--sp];
                if (__uint_as_float((unsigned)(e >> 32)) <= tBest) { ref = (int)(unsigned)e; return true; }
            }
            return false;
        };
        for (;;) {
            while (ref >= 0) {
                if (++iters > kIterBudget) { err |= DEV_ERR_BUDGET; return -1; }
                const GNode4* np = S.nodes8[ref].q;
                float t[8];
                bool hh[8];
                int c[8];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const GNode4* q = np + h;
                    const float4 nx = plane(q, onx), fx = plane(q, ofx), ny = plane(q, ony), fy = plane(q, ofy);
                    const float4 nz = plane(q, onz), fz = plane(q, ofz);
                    const int4 ch = __ldg(&q->child);
                    float th[4];
                    bool hk[4];
                    slab4_nh(nx, fx, ny, fy, nz, fz, R2, tMin, tBest, th, hk);
                    t[4 * h] = th[0]; t[4 * h + 1] = th[1]; t[4 * h + 2] = th[2]; t[4 * h + 3] = th[3];
                    hh[4 * h] = hk[0]; hh[4 * h + 1] = hk[1]; hh[4 * h + 2] = hk[2]; hh[4 * h + 3] = hk[3];
                    c[4 * h] = ch.x; c[4 * h + 1] = ch.y; c[4 * h + 2] = ch.z; c[4 * h + 3] = ch.w;
                }
                int nh = 0;
#pragma unroll
                for (int k = 0; k < 8; ++k) nh += int(hh[k]);
                if (nh == 1) {
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        if (hh[k]) ref = c[k];
                } else if (nh > 1) {
                    const float inf = __int_as_float(0x7f800000);
#pragma unroll
                    for (int k = 0; k < 8; ++k) t[k] = hh[k] ? t[k] : inf;
                    float* t0 = t;
                    float* t1 = t + 4;
                    int* c0 = c;
                    int* c1 = c + 4;
                    sort4(*reinterpret_cast<float(*)[4]>(t0), *reinterpret_cast<int(*)[4]>(c0));
                    sort4(*reinterpret_cast<float(*)[4]>(t1), *reinterpret_cast<int(*)[4]>(c1));
                    // odd-even merge of the two sorted halves
                    cswap(t[0], c[0], t[4], c[4]);
                    cswap(t[1], c[1], t[5], c[5]);
                    cswap(t[2], c[2], t[6], c[6]);
                    cswap(t[3], c[3], t[7], c[7]);
                    cswap(t[2], c[2], t[4], c[4]);
                    cswap(t[3], c[3], t[5], c[5]);
                    cswap(t[1], c[1], t[2], c[2]);
                    cswap(t[3], c[3], t[4], c[4]);
                    cswap(t[5], c[5], t[6], c[6]);
#pragma unroll
                    for (int k = 7; k >= 1; --k)
                        if (t[k] <= tBest) push(c[k], t[k]);
                    ref = c[0];
                } else if (!pop()) {
                    return best;
                }
            }
            do {
                if (++iters > kIterBudget) { err |= DEV_ERR_BUDGET; return -1; }
                const int code = ~ref;
                const int first = code >> 4, cnt = code & 15;
                switch (wr.kz) {
                    case 0: leaf_wt<0>(S.tris, S.tie, first, cnt, o, wr, tMin, tBest, best); break;
                    case 1: leaf_wt<1>(S.tris, S.tie, first, cnt, o, wr, tMin, tBest, best); break;
                    default: leaf_wt<2>(S.tris, S.tie, first, cnt, o, wr, tMin, tBest, best); break;
                }
                if (!pop()) return best;
            } while (ref < 0);
        }
    }
};

// Speculative variant of Walker<false>::closest with the watertight test (Aila and
// Laine, "Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009): a lane
// that reaches a leaf parks it and keeps walking inner nodes (pruning with its not
// yet lowered closest distance) until every lane of `mask` holds a parked leaf or
// has emptied its stack; then all lanes test their leaves.  Every lane of `mask`
// calls it together and leaves it together (each runs the same sequence of
// __any_sync); a lane whose iteration budget runs out stops walking but stays in
// step, and returns -1 with DEV_ERR_BUDGET.
__device__ __forceinline__ int closest_speculative(const SceneView& S, F3 o, F3 d, float tMin, float& tBest,
                                                   uint32_t& err, unsigned mask) {
    const F3 inv{slab_inv(d.x), slab_inv(d.y), slab_inv(d.z)};
    const WtRay wr = wt_ray(d);
    const F3 oi{o.x * inv.x, o.y * inv.y, o.z * inv.z};
    const Slab2 R2 = slab2(inv, oi);
    const unsigned onx = inv.x < 0.0f ? 16u : 0u, ony = inv.y < 0.0f ? 48u : 32u, onz = inv.z < 0.0f ? 80u : 64u;
    const unsigned ofx = onx ^ 16u, ofy = ony ^ 16u, ofz = onz ^ 16u;
    unsigned long long stack[kStackDepth];
    int sp = 0;
    int ref = 0;        // current entry: inner node (>= 0) or leaf (< 0), valid while `has`
    bool has = true;
    int parked = 0;     // a leaf waiting to be tested (< 0), or 0
    int best = -1;
    bool over = false;
    uint32_t iters = 0;
    auto plane = [](const GNode4* p, unsigned off) {
        return __ldg(reinterpret_cast<const float4*>(reinterpret_cast<const char*>(p) + off));
    };
    auto push = [&](int r, float t) {
        if (sp < kStackDepth) stack[sp++] = pack_entry(r, t);
        else err |= DEV_ERR_STACK;
    };
    auto pop = [&]() {
        while (sp > 0) {
            const unsigned long long e = stack[--sp];
            if (__uint_as_float((unsigned)(e >> 32)) <= tBest) { ref = (int)(unsigned)e; return true; }
        }
        return false;
    };
    auto test_leaf = [&](int leaf) {
        const int code = ~leaf;
        const int first = code >> 4, cnt = code & 15;
        switch (wr.kz) {
            case 0: leaf_wt<0>(S.tris, S.tie, first, cnt, o, wr, tMin, tBest, best); break;
            case 1: leaf_wt<1>(S.tris, S.tie, first, cnt, o, wr, tMin, tBest, best); break;
            default: leaf_wt<2>(S.tris, S.tie, first, cnt, o, wr, tMin, tBest, best); break;
        }
    };
    for (;;) {
        // inner nodes, while some lane holds an entry but no parked leaf
        while (__any_sync(mask, has && parked == 0)) {
            if (has && ref >= 0) {
                if (++iters > kIterBudget) {
                    over = true;
                    has = false;
                    parked = 0;
                } else {
                    const GNode4* np = S.nodes + ref;
                    const float4 nx = plane(np, onx), fx = plane(np, ofx), ny = plane(np, ony), fy = plane(np, ofy);
                    const float4 nz = plane(np, onz), fz = plane(np, ofz);
                    const int4 ch = __ldg(&np->child);
                    float t[4];
                    bool hh[4];
                    slab4_nh(nx, fx, ny, fy, nz, fz, R2, tMin, tBest, t, hh);
                    const bool h0 = hh[0], h1 = hh[1], h2 = hh[2], h3 = hh[3];
                    int c[4] = {ch.x, ch.y, ch.z, ch.w};
                    const int nh = int(h0) + int(h1) + int(h2) + int(h3);
                    if (nh == 1) {
                        ref = h0 ? c[0] : h1 ? c[1] : h2 ? c[2] : c[3];
                    } else if (nh == 2) {
                        const float ta = h0 ? t[0] : h1 ? t[1] : t[2];
                        const int ca = h0 ? c[0] : h1 ? c[1] : c[2];
                        const float tb = h3 ? t[3] : h2 ? t[2] : t[1];
                        const int cb = h3 ? c[3] : h2 ? c[2] : c[1];
                        const bool sw = tb < ta;
                        push(sw ? ca : cb, sw ? ta : tb);
                        ref = sw ? cb : ca;
                    } else if (nh > 2) {
                        const float inf = __int_as_float(0x7f800000);
                        t[0] = h0 ? t[0] : inf;
                        t[1] = h1 ? t[1] : inf;
                        t[2] = h2 ? t[2] : inf;
                        t[3] = h3 ? t[3] : inf;
                        sort4(t, c);
                        if (t[3] <= tBest) push(c[3], t[3]);
                        if (t[2] <= tBest) push(c[2], t[2]);
                        push(c[1], t[1]);
                        ref = c[0];
                    } else {
                        has = pop();
                    }
                }
            }
            if (has && ref < 0 && parked == 0) {  // a leaf: park it and walk on
                parked = ref;
                has = pop();
            }
        }
        // leaves: the parked one, then this lane's run of leaf entries
        if (parked != 0) {
            test_leaf(parked);
            parked = 0;
        }
        while (has && ref < 0) {
            if (++iters > kIterBudget) {
                over = true;
                has = false;
                break;
            }
            test_leaf(ref);
            has = pop();
        }
        if (!__any_sync(mask, has)) break;
    }
    if (over) {
        err |= DEV_ERR_BUDGET;
        return -1;
    }
    return best;
}

template <>
struct Walker<true> {
    __device__ __forceinline__ static int closest(const SceneView& S, D3 o, D3 d, double tMin, double& tBest,
                                                  uint32_t& err) {
        const D3 inv{slab_inv(d.x), slab_inv(d.y), slab_inv(d.z)};
        unsigned long long stack[kStackDepth];
        int sp = 0;
        int ref = 0;
        int best = -1;
        uint32_t iters = 0;
        // entry distances are stored rounded down to float, so the pruning test
        // (entry <= tBest) stays conservative
        auto push = [&](int r, double t) {
            if (sp < kStackDepth) stack[sp++] = pack_entry(r, __double2float_rd(t));
            else err |= DEV_ERR_STACK;
        };
        auto pop = [&]() {
            while (sp > 0) {
                const unsigned long long e = stack[--sp];
                if (double(__uint_as_float((unsigned)(e >> 32))) <= tBest) { ref = (int)(unsigned)e; return true; }
            }
            return false;
        };
        for (;;) {
            while (ref >= 0) {
                if (++iters > kIterBudget) { err |= DEV_ERR_BUDGET; return -1; }
                const GNode4 n = load_node(S.nodes + ref);
                double t[4] = {slab_d(n.lox.x, n.hix.x, n.loy.x, n.hiy.x, n.loz.x, n.hiz.x, o, inv, tMin, tBest),
                               slab_d(n.lox.y, n.hix.y, n.loy.y, n.hiy.y, n.loz.y, n.hiz.y, o, inv, tMin, tBest),
                               slab_d(n.lox.z, n.hix.z, n.loy.z, n.hiy.z, n.loz.z, n.hiz.z, o, inv, tMin, tBest),
                               slab_d(n.lox.w, n.hix.w, n.loy.w, n.hiy.w, n.loz.w, n.hiz.w, o, inv, tMin, tBest)};
                int c[4] = {n.child.x, n.child.y, n.child.z, n.child.w};
                // most visits accept exactly one child (no ordering needed); two or
                // more are sorted and all but the nearest pushed, farthest first
                const bool h0 = t[0] <= tBest, h1 = t[1] <= tBest, h2 = t[2] <= tBest, h3 = t[3] <= tBest;
                const int nh = int(h0) + int(h1) + int(h2) + int(h3);
                if (nh == 1) {
                    ref = h0 ? c[0] : h1 ? c[1] : h2 ? c[2] : c[3];
                } else if (nh > 1) {
                    sort4(t, c);
                    if (t[3] <= tBest) push(c[3], t[3]);
                    if (t[2] <= tBest) push(c[2], t[2]);
                    push(c[1], t[1]);
                    ref = c[0];
                } else if (!pop()) {
                    return best;
                }
            }
            do {
                if (++iters > kIterBudget) { err |= DEV_ERR_BUDGET; return -1; }
                const int code = ~ref;
                const int first = code >> 4, cnt = code & 15;
                for (int k = 0; k < cnt; ++k) {
                    double tt;
                    if (mt_d(S.tris64[first + k], o, d, tMin, tBest, tt) && replaces(tt, first + k, tBest, best, S.tie)) {
                        tBest = tt;
                        best = first + k;
                    }
                }
                if (!pop()) return best;
            } while (ref < 0);
        }
    }
};

// Segment owning a work item: base[] holds each segment's first item (ascending).
__device__ __forceinline__ int find_segment(const int64_t* base, int n, int64_t item) {
    int lo = 0, hi = n;  // base[lo] <= item < base[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(base + mid) <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

}  // namespace sbr
