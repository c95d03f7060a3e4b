// sbr_oracle.cpp -- CPU restatement of SagittaSBR's hot path, used ONLY as test
// infrastructure (tests/, the smoke check and bench.py's cpu_baseline leg).
// Nothing in the product links or calls this file.
//
// It restates, in FP64 (or FP32 through the template parameter), the exact
// arithmetic of the reference path so that GPU results can be checked against it:
//
//   launcher frame per angle ........ src/app/sweep.cu:336-364
//   angle grid from config .......... src/app/sweep.cu:339-347
//   ray origin per pixel ............ src/cuda/rtKernels.cu:118-123
//   bounce loop, reflect, nudge ..... src/cuda/rtKernels.cu:126-158
//   Moller-Trumbore test ............ src/cuda/rtKernels.cu:10-44
//   slab test ....................... src/cuda/rtKernels.cu:46-61
//   binary BVH walk (64-deep stack) . src/cuda/rtKernels.cu:63-100
//   PO exit-ray term ................ src/cuda/poKernels.cu:81-109
//   k, ray area ..................... src/app/sweep.cu:50-55
//   sigma, dBsm ..................... src/app/sweep.cu:228-231
//   binned SAH build (16 bins, leaf 4, median fallback) src/scene/bvhBuilder.cpp:93-360
//
// Operation order follows the reference (vec3 helpers in include/RT/vec3.h:48-174),
// and the library is built with -ffp-contract=off, so the FP64 restatement is
// bit-comparable with the reference's own per-ray routine compiled for the host
// (oracle/_ref).  Two accelerations are offered: the reference SAH tree walked in
// the reference order (counts box and triangle tests for the roofline), and brute
// force over all triangles in index order, which also reports per-ray ambiguity
// flags (edge, grazing-threshold, t-tie and tMin proximity) used to exclude
// ill-conditioned rays from hit-sequence comparisons.
//
// The field sum is deterministic: each ray row is summed in index order, rows are
// summed in order, in FP64 whatever the traversal precision.

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <class R>
struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline V3<R> mulv(V3<R> a, V3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> inline V3<R> scale(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline V3<R> divs(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, -(a.x * b.z - a.z * b.x), a.x * b.y - a.y * b.x};
}
template <class R> inline R length(V3<R> a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
template <class R> inline V3<R> unit(V3<R> a) { return divs(a, length(a)); }
template <class R> inline V3<R> vmin(V3<R> a, V3<R> b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
template <class R> inline V3<R> vmax(V3<R> a, V3<R> b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }

template <class R> struct Lim;
template <> struct Lim<float> { static float big() { return FLT_MAX; } };
template <> struct Lim<double> { static double big() { return 1.7976931348623158e+308; } };

template <class R>
struct Tri {
    V3<R> v0, v1, v2;
    int32_t id;  // index in the caller's triangle list
};

template <class R>
struct Node {
    V3<R> lo, hi;
    int32_t left, right, first, count;
};

// ---------------------------------------------------------------- SAH build
// Restates src/scene/bvhBuilder.cpp:22-312 (sequential: node ids are handed out in
// pre-order, which is the order the reference produces with enableParallel=false).
template <class R>
struct TreeBuilder {
    std::vector<Tri<R>>& tris;
    std::vector<Node<R>> nodes;
    int counter = 0;
    int leafSize = 4;
    int binCount = 16;

    explicit TreeBuilder(std::vector<Tri<R>>& t) : tris(t) {}

    static V3<R> tmin3(const Tri<R>& t) { return vmin(vmin(t.v0, t.v1), t.v2); }
    static V3<R> tmax3(const Tri<R>& t) { return vmax(vmax(t.v0, t.v1), t.v2); }
    static V3<R> centroid(const Tri<R>& t) { return divs(t.v0 + t.v1 + t.v2, R(3.0)); }
    static R area(V3<R> lo, V3<R> hi) {
        V3<R> d = hi - lo;
        R dx = std::fmax(R(0), d.x), dy = std::fmax(R(0), d.y), dz = std::fmax(R(0), d.z);
        return R(2.0) * (dx * dy + dy * dz + dz * dx);
    }
    static int widest(V3<R> v) {
        if (v.x >= v.y && v.x >= v.z) return 0;
        if (v.y >= v.z) return 1;
        return 2;
    }
    void bounds(int s, int e, V3<R>& lo, V3<R>& hi) const {
        R B = Lim<R>::big();
        lo = {B, B, B};
        hi = {-B, -B, -B};
        for (int i = s; i < e; ++i) { lo = vmin(lo, tmin3(tris[i])); hi = vmax(hi, tmax3(tris[i])); }
    }
    void cbounds(int s, int e, V3<R>& lo, V3<R>& hi) const {
        R B = Lim<R>::big();
        lo = {B, B, B};
        hi = {-B, -B, -B};
        for (int i = s; i < e; ++i) { V3<R> c = centroid(tris[i]); lo = vmin(lo, c); hi = vmax(hi, c); }
    }
    bool split_median(int s, int e, int& mid) {
        V3<R> clo, chi;
        cbounds(s, e, clo, chi);
        int ax = widest(chi - clo);
        mid = s + (e - s) / 2;
        std::nth_element(tris.begin() + s, tris.begin() + mid, tris.begin() + e,
                         [ax](const Tri<R>& a, const Tri<R>& b) { return centroid(a)[ax] < centroid(b)[ax]; });
        return mid > s && mid < e;
    }
    bool split_sah(int s, int e, V3<R> lo, V3<R> hi, int& mid) {
        struct Bin { V3<R> lo, hi; int n; };
        const R B = Lim<R>::big();
        int n = e - s;
        V3<R> clo, chi;
        cbounds(s, e, clo, chi);
        V3<R> cext = chi - clo;
        R parent = area(lo, hi);
        if (parent <= R(0)) return false;
        int bestAx = -1, bestSplit = -1;
        R bestCost = B;
        std::vector<Bin> bins(binCount);
        std::vector<V3<R>> llo(binCount), lhi(binCount), rlo(binCount), rhi(binCount);
        std::vector<int> ln(binCount), rn(binCount);
        for (int ax = 0; ax < 3; ++ax) {
            R ext = cext[ax];
            if (ext <= R(1.0e-6)) continue;
            for (auto& b : bins) { b.lo = {B, B, B}; b.hi = {-B, -B, -B}; b.n = 0; }
            for (int i = s; i < e; ++i) {
                R off = (centroid(tris[i])[ax] - clo[ax]) / ext;
                int bi = static_cast<int>(off * binCount);
                bi = bi < 0 ? 0 : (bi >= binCount ? binCount - 1 : bi);
                bins[bi].lo = vmin(bins[bi].lo, tmin3(tris[i]));
                bins[bi].hi = vmax(bins[bi].hi, tmax3(tris[i]));
                bins[bi].n += 1;
            }
            V3<R> rl{B, B, B}, rh{-B, -B, -B};
            int rc = 0;
            for (int i = 0; i < binCount; ++i) {
                if (bins[i].n > 0) { rl = vmin(rl, bins[i].lo); rh = vmax(rh, bins[i].hi); rc += bins[i].n; }
                llo[i] = rl; lhi[i] = rh; ln[i] = rc;
            }
            rl = {B, B, B}; rh = {-B, -B, -B}; rc = 0;
            for (int i = binCount - 1; i >= 0; --i) {
                if (bins[i].n > 0) { rl = vmin(rl, bins[i].lo); rh = vmax(rh, bins[i].hi); rc += bins[i].n; }
                rlo[i] = rl; rhi[i] = rh; rn[i] = rc;
            }
            for (int i = 0; i < binCount - 1; ++i) {
                int a = ln[i], b = rn[i + 1];
                if (a == 0 || b == 0) continue;
                R cost = (area(llo[i], lhi[i]) * a + area(rlo[i + 1], rhi[i + 1]) * b) / parent;
                if (cost < bestCost) { bestCost = cost; bestAx = ax; bestSplit = i; }
            }
        }
        if (bestAx < 0) return false;
        if (bestCost >= static_cast<R>(n)) return false;
        R ext = cext[bestAx];
        if (ext <= R(1.0e-6)) return false;
        R pos = clo[bestAx] + ext * (static_cast<R>(bestSplit + 1) / static_cast<R>(binCount));
        auto it = std::partition(tris.begin() + s, tris.begin() + e,
                                 [bestAx, pos](const Tri<R>& t) { return centroid(t)[bestAx] < pos; });
        mid = static_cast<int>(it - tris.begin());
        return mid > s && mid < e;
    }
    int build(int s, int e) {
        V3<R> lo, hi;
        bounds(s, e, lo, hi);
        int idx = counter++;
        nodes[idx] = Node<R>{lo, hi, -1, -1, s, e - s};
        if (e - s <= leafSize) return idx;
        int mid = -1;
        bool ok = split_sah(s, e, lo, hi, mid);
        if (!ok) ok = split_median(s, e, mid);
        if (!ok) return idx;
        int l = build(s, mid);
        int r = build(mid, e);
        nodes[idx].left = l;
        nodes[idx].right = r;
        nodes[idx].first = 0;
        nodes[idx].count = 0;
        return idx;
    }
    void run() {
        if (tris.empty()) return;
        nodes.assign(tris.size() * 2 - 1, Node<R>{});
        counter = 0;
        build(0, static_cast<int>(tris.size()));
        nodes.resize(counter);
    }
};

// --------------------------------------------------------------- intersection
template <class R>
struct Hit {
    R t;
    V3<R> p, n;
    int32_t id;
};

// Moller-Trumbore, two-sided, |det| < 1e-6 rejected, inclusive bounds
// (src/cuda/rtKernels.cu:10-44).
template <class R>
inline bool mt_hit(const Tri<R>& tri, V3<R> o, V3<R> d, R tMin, R tMax, Hit<R>& h) {
    const R eps = R(1.0e-6);
    V3<R> e1 = tri.v1 - tri.v0;
    V3<R> e2 = tri.v2 - tri.v0;
    V3<R> pv = cross(d, e2);
    R det = dot(e1, pv);
    if (std::fabs(det) < eps) return false;
    R inv = R(1.0) / det;
    V3<R> tv = o - tri.v0;
    R u = dot(tv, pv) * inv;
    if (u < R(0) || u > R(1)) return false;
    V3<R> qv = cross(tv, e1);
    R v = dot(d, qv) * inv;
    if (v < R(0) || u + v > R(1)) return false;
    R t = dot(e2, qv) * inv;
    if (t < tMin || t > tMax) return false;
    h.t = t;
    h.p = o + scale(t, d);
    h.n = unit(cross(e1, e2));
    h.id = tri.id;
    return true;
}

// Slab test with the reciprocal recomputed per node (src/cuda/rtKernels.cu:46-61).
template <class R>
inline bool slab(const Node<R>& nd, V3<R> o, V3<R> d, R tMin, R tMax) {
    V3<R> inv(R(1.0) / d.x, R(1.0) / d.y, R(1.0) / d.z);
    V3<R> t0 = mulv(nd.lo - o, inv);
    V3<R> t1 = mulv(nd.hi - o, inv);
    R tmin = std::fmax(std::fmax(std::fmin(t0.x, t1.x), std::fmin(t0.y, t1.y)), std::fmin(t0.z, t1.z));
    R tmax = std::fmin(std::fmin(std::fmax(t0.x, t1.x), std::fmax(t0.y, t1.y)), std::fmax(t0.z, t1.z));
    tmin = std::fmax(tmin, tMin);
    tmax = std::fmin(tmax, tMax);
    return tmax >= tmin;
}

struct Counters {
    uint64_t box = 0, tri = 0;
};

// Reference walk order: pop, test box against the current closest t, leaf -> test
// its triangles in order, inner -> push left then right (right is visited first).
template <class R>
inline bool walk_tree(const std::vector<Tri<R>>& tris, const std::vector<Node<R>>& nodes, V3<R> o, V3<R> d,
                      R tMin, R tMax, Hit<R>& rec, Counters& c) {
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    bool any = false;
    R closest = tMax;
    Hit<R> tmp;
    while (sp > 0) {
        const Node<R>& nd = nodes[stack[--sp]];
        c.box++;
        if (!slab(nd, o, d, tMin, closest)) continue;
        if (nd.count > 0) {
            for (int i = 0; i < nd.count; ++i) {
                c.tri++;
                if (mt_hit(tris[nd.first + i], o, d, tMin, closest, tmp)) { any = true; closest = tmp.t; rec = tmp; }
            }
        } else if (sp + 2 <= 64) {
            stack[sp++] = nd.left;
            stack[sp++] = nd.right;
        }
    }
    return any;
}

template <class R>
inline bool walk_all(const std::vector<Tri<R>>& tris, V3<R> o, V3<R> d, R tMin, R tMax, Hit<R>& rec, Counters& c) {
    bool any = false;
    R closest = tMax;
    Hit<R> tmp;
    for (const auto& t : tris) {
        c.tri++;
        if (mt_hit(t, o, d, tMin, closest, tmp)) { any = true; closest = tmp.t; rec = tmp; }
    }
    return any;
}

// Ambiguity flags (FP64 recomputation over every triangle): a decision of the
// closest-hit query lies within the given tolerance of flipping.
enum : int32_t { AMB_EDGE = 1, AMB_DET = 2, AMB_TIE = 4, AMB_TMIN = 8 };

template <class R>
int32_t ambiguity(const std::vector<Tri<R>>& tris, V3<R> oR, V3<R> dR, bool hit, const Hit<R>& best, double tMin,
                  double dEdge, double dT, double dDet) {
    V3<double> o(oR.x, oR.y, oR.z), d(dR.x, dR.y, dR.z);
    double tBest = hit ? double(best.t) : std::numeric_limits<double>::infinity();
    int32_t flags = 0;
    for (const auto& T : tris) {
        V3<double> a(T.v0.x, T.v0.y, T.v0.z), b(T.v1.x, T.v1.y, T.v1.z), c(T.v2.x, T.v2.y, T.v2.z);
        V3<double> e1 = b - a, e2 = c - a;
        V3<double> pv = cross(d, e2);
        double det = dot(e1, pv);
        if (std::fabs(det) < 1e-300) continue;
        V3<double> tv = o - a;
        double u = dot(tv, pv) / det;
        V3<double> qv = cross(tv, e1);
        double v = dot(d, qv) / det;
        double t = dot(e2, qv) / det;
        if (!(t >= tMin - dT && t <= tBest + dT)) continue;
        double a2 = length(cross(e1, e2));
        double lab = length(e1), lac = length(e2), lbc = length(c - b);
        if (a2 <= 0 || lab <= 0 || lac <= 0 || lbc <= 0) continue;
        double w = 1.0 - u - v;
        double s = std::fmin(std::fmin(w * a2 / lbc, u * a2 / lac), v * a2 / lab);
        if (std::fabs(s) <= dEdge) { flags |= AMB_EDGE; continue; }
        if (s < 0) continue;
        if (std::fabs(std::fabs(det) - 1e-6) <= dDet * 1e-6) flags |= AMB_DET;
        if (std::fabs(det) < 1e-6 * (1.0 - dDet)) continue;
        if (std::fabs(t - tMin) <= dT) flags |= AMB_TMIN;
        if (hit && T.id != best.id && std::fabs(t - tBest) <= dT) flags |= AMB_TIE;
    }
    return flags;
}

}  // namespace

extern "C" {

// Per-ray record written by oracle_sweep when requested (layout mirrored in tests).
#define ORACLE_MAX_REC 16
typedef struct oracle_ray {
    int32_t count;       // successful reflections (hitCount)
    int32_t amb;         // ambiguity flags OR-ed over all queries (brute force only)
    double dist;         // summed path from the launcher plane
    double normal[3];    // last hit normal
    double lastdir[3];   // incoming direction of the last hit
    int32_t tri[ORACLE_MAX_REC];  // triangle ids of the first hits, -1 padded
} oracle_ray;

typedef struct oracle_counts {
    uint64_t rays;        // rays traced
    uint64_t hit_rays;    // rays with count > 0
    uint64_t bounces;     // sum of counts
    uint64_t queries;     // closest-hit queries
    uint64_t box_tests;   // slab tests (tree walk only)
    uint64_t tri_tests;   // triangle tests
} oracle_counts;

int oracle_ray_record_size(void) { return (int)sizeof(oracle_ray); }
int oracle_max_rec(void) { return ORACLE_MAX_REC; }

}  // extern "C"

namespace {

template <class R>
struct Frame {
    V3<R> dir, rayDir, u, v, llc;
};

// src/app/sweep.cu:342-364 (angles in degrees, converted in R precision).
template <class R>
Frame<R> make_frame(double thetaDeg, double phiDeg, R G) {
    const R pi = R(M_PI);
    R th = R(thetaDeg) * pi / R(180.0);
    R ph = R(phiDeg) * pi / R(180.0);
    Frame<R> f;
    f.dir = V3<R>(std::sin(th) * std::cos(ph), std::sin(th) * std::sin(ph), std::cos(th));
    f.rayDir = -f.dir;
    V3<R> up(0, 1, 0);
    if (std::fabs(f.dir.y) > R(0.99)) up = V3<R>(1, 0, 0);
    f.u = scale(G, unit(cross(up, f.dir)));
    f.v = scale(G, unit(cross(f.dir, f.u)));
    f.llc = scale(R(10.0) * G, f.dir) - scale(R(0.5), f.u) - scale(R(0.5), f.v);
    return f;
}

// Origin of the ray of pixel (i, j) on an nx x ny launcher (src/cuda/rtKernels.cu:118-123).
template <class R>
V3<R> ray_origin(const Frame<R>& fr, int32_t i, int32_t j, int32_t nx, int32_t ny) {
    R u = (R(i) + R(0.5)) / R(nx);
    R v = (R(j) + R(0.5)) / R(ny);
    return fr.llc + scale(u, fr.u) + scale(v, fr.v);
}

// What one ray leaves after its bounce loop.
template <class R>
struct RayTrace {
    int32_t count = 0;  // successful reflections
    int32_t amb = 0;    // ambiguity flags OR-ed over the queries (brute force with wantAmb)
    R dist = R(0);      // summed path
    V3<R> nLast, dLast;
    int32_t ids[ORACLE_MAX_REC];
    uint64_t queries = 0;
};

// The bounce loop of one ray (src/cuda/rtKernels.cu:126-158): closest hit with
// tMin = 1e-3, reflect, nudge 1e-4 along the normal, stop on a miss.
template <class R>
void trace_ray(const std::vector<Tri<R>>& tris, const std::vector<Node<R>>& nodes, const std::vector<Tri<R>>& original,
               int32_t accel, bool wantAmb, V3<R> o, V3<R> d, int32_t maxBounces, double dEdge, double dT, double dDet,
               RayTrace<R>& rt, Counters& cnt) {
    const R tMin = R(0.001), tMax = R(1e20), nudge = R(1e-4);
    for (int q = 0; q < ORACLE_MAX_REC; ++q) rt.ids[q] = -1;
    for (int32_t b = 0; b < maxBounces; ++b) {
        Hit<R> h;
        rt.queries++;
        bool hit = accel == 1 ? walk_tree(tris, nodes, o, d, tMin, tMax, h, cnt)
                              : walk_all(original, o, d, tMin, tMax, h, cnt);
        if (wantAmb && accel == 0) rt.amb |= ambiguity(original, o, d, hit, h, double(tMin), dEdge, dT, dDet);
        if (!hit) break;
        rt.nLast = h.n;
        rt.dLast = d;
        if (rt.count < ORACLE_MAX_REC) rt.ids[rt.count] = h.id;
        rt.count++;
        rt.dist += h.t;
        d = unit(d - scale(R(2.0) * dot(d, h.n), h.n));
        o = h.p + scale(nudge, h.n);
    }
}

template <class R>
int sweep_impl(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
               const double* thetaDeg, const double* phiDeg, int64_t nAngles, const double* freqHz,
               int64_t nFreqs, int32_t nx, int32_t ny, double gridSize, int32_t maxBounces, double reflConst,
               int32_t accel, int32_t nThreads, double* outRe, double* outIm, oracle_counts* counts,
               oracle_ray* rays, double dEdge, double dT, double dDet) {
    if (ntris <= 0 || nverts <= 0 || nx <= 0 || ny <= 0 || nAngles < 0 || nFreqs <= 0) return 1;
    std::vector<Tri<R>> tris(ntris);
    const R sc = R(modelScale);
    for (int64_t i = 0; i < ntris; ++i) {
        uint32_t a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        if (a >= nverts || b >= nverts || c >= nverts) return 2;
        auto P = [&](uint32_t k) { return V3<R>(R(xyz[3 * k]) * sc, R(xyz[3 * k + 1]) * sc, R(xyz[3 * k + 2]) * sc); };
        tris[i] = Tri<R>{P(a), P(b), P(c), (int32_t)i};
    }
    std::vector<Tri<R>> original = tris;  // index order, for brute force and ambiguity
    TreeBuilder<R> tb(tris);
    if (accel == 1) tb.run();

#ifdef _OPENMP
    if (nThreads > 0) omp_set_num_threads(nThreads);
#endif
    const R G = R(gridSize);
    const R c0 = R(299792458.0);
    const R rayArea = (G * G) / R(int64_t(nx) * int64_t(ny));
    std::vector<R> kk(nFreqs);
    for (int64_t f = 0; f < nFreqs; ++f) kk[f] = R(2.0) * R(M_PI) / (c0 / R(freqHz[f]));
    const R twoPi = R(2.0) * R(M_PI);
    const R fourPi = R(4.0) * R(M_PI);

    std::vector<double> rowRe((size_t)ny * nFreqs), rowIm((size_t)ny * nFreqs);
    for (int64_t a = 0; a < nAngles; ++a) {
        Frame<R> fr = make_frame<R>(thetaDeg[a], phiDeg[a], G);
        std::atomic<uint64_t> cHit{0}, cBounce{0}, cQuery{0}, cBox{0}, cTri{0};
#pragma omp parallel for schedule(dynamic)
        for (int32_t j = 0; j < ny; ++j) {
            Counters cnt;
            uint64_t hitRays = 0, bounces = 0, queries = 0;
            std::vector<double> accRe(nFreqs, 0.0), accIm(nFreqs, 0.0);
            for (int32_t i = 0; i < nx; ++i) {
                RayTrace<R> rt;
                trace_ray(tris, tb.nodes, original, accel, rays != nullptr, ray_origin(fr, i, j, nx, ny), fr.rayDir,
                          maxBounces, dEdge, dT, dDet, rt, cnt);
                queries += rt.queries;
                const int32_t count = rt.count, amb = rt.amb;
                const R dist = rt.dist;
                const V3<R> nLast = rt.nLast, dLast = rt.dLast;
                const int32_t* ids = rt.ids;
                if (count > 0) {
                    hitRays++;
                    bounces += (uint64_t)count;
                    R Rn = R(1.0);
                    for (int32_t b = 0; b < count; ++b) Rn *= R(reflConst);
                    R cosT = dot(nLast, -dLast);
                    if (cosT > R(0)) {
                        for (int64_t f = 0; f < nFreqs; ++f) {
                            R k = kk[f];
                            R phase = R(2.0) * k * dist;
                            phase = std::fmod(phase, twoPi);
                            R mag = (k * rayArea / fourPi) * R(2.0) * cosT * Rn;
                            R s = std::sin(phase), c = std::cos(phase);
                            accRe[f] += double(-mag * s);
                            accIm[f] += double(mag * c);
                        }
                    }
                }
                if (rays) {
                    oracle_ray& rr = rays[(size_t)a * nx * ny + (size_t)j * nx + i];
                    rr.count = count;
                    rr.amb = amb;
                    rr.dist = double(dist);
                    rr.normal[0] = count ? double(nLast.x) : 0.0;
                    rr.normal[1] = count ? double(nLast.y) : 0.0;
                    rr.normal[2] = count ? double(nLast.z) : 0.0;
                    rr.lastdir[0] = count ? double(dLast.x) : 0.0;
                    rr.lastdir[1] = count ? double(dLast.y) : 0.0;
                    rr.lastdir[2] = count ? double(dLast.z) : 0.0;
                    for (int q = 0; q < ORACLE_MAX_REC; ++q) rr.tri[q] = ids[q];
                }
            }
            for (int64_t f = 0; f < nFreqs; ++f) {
                rowRe[(size_t)j * nFreqs + f] = accRe[f];
                rowIm[(size_t)j * nFreqs + f] = accIm[f];
            }
            cHit += hitRays;
            cBounce += bounces;
            cQuery += queries;
            cBox += cnt.box;
            cTri += cnt.tri;
        }
        for (int64_t f = 0; f < nFreqs; ++f) {
            double re = 0, im = 0;
            for (int32_t j = 0; j < ny; ++j) { re += rowRe[(size_t)j * nFreqs + f]; im += rowIm[(size_t)j * nFreqs + f]; }
            outRe[a * nFreqs + f] = re;
            outIm[a * nFreqs + f] = im;
        }
        if (counts) {
            counts[a].rays = (uint64_t)nx * (uint64_t)ny;
            counts[a].hit_rays = cHit;
            counts[a].bounces = cBounce;
            counts[a].queries = cQuery;
            counts[a].box_tests = cBox;
            counts[a].tri_tests = cTri;
        }
    }
    return 0;
}

// Explicit ray list: ray k is pixel (i, j) = (rays[3k+1], rays[3k+2]) of the nx x ny
// launcher of angle rays[3k], traced as oracle_sweep traces it.  One record per ray
// (ambiguity flags with brute force) and the totals over the list in counts[0].
template <class R>
int trace_list_impl(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
                    const double* thetaDeg, const double* phiDeg, int64_t nAngles, const int32_t* rayList,
                    int64_t nRays, int32_t nx, int32_t ny, double gridSize, int32_t maxBounces, int32_t accel,
                    int32_t nThreads, oracle_ray* rays, oracle_counts* counts, double dEdge, double dT, double dDet) {
    if (ntris <= 0 || nverts <= 0 || nx <= 0 || ny <= 0 || nAngles <= 0 || nRays < 0) return 1;
    for (int64_t k = 0; k < nRays; ++k) {
        const int32_t a = rayList[3 * k], i = rayList[3 * k + 1], j = rayList[3 * k + 2];
        if (a < 0 || a >= nAngles || i < 0 || i >= nx || j < 0 || j >= ny) return 3;
    }
    std::vector<Tri<R>> tris(ntris);
    const R sc = R(modelScale);
    for (int64_t i = 0; i < ntris; ++i) {
        uint32_t a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        if (a >= nverts || b >= nverts || c >= nverts) return 2;
        auto P = [&](uint32_t k) { return V3<R>(R(xyz[3 * k]) * sc, R(xyz[3 * k + 1]) * sc, R(xyz[3 * k + 2]) * sc); };
        tris[i] = Tri<R>{P(a), P(b), P(c), (int32_t)i};
    }
    std::vector<Tri<R>> original = tris;
    TreeBuilder<R> tb(tris);
    if (accel == 1) tb.run();
#ifdef _OPENMP
    if (nThreads > 0) omp_set_num_threads(nThreads);
#endif
    std::vector<Frame<R>> frames(nAngles);
    for (int64_t a = 0; a < nAngles; ++a) frames[a] = make_frame<R>(thetaDeg[a], phiDeg[a], R(gridSize));
    std::atomic<uint64_t> cHit{0}, cBounce{0}, cQuery{0}, cBox{0}, cTri{0};
#pragma omp parallel
    {
        Counters cnt;
        uint64_t hitRays = 0, bounces = 0, queries = 0;
#pragma omp for schedule(dynamic, 16)
        for (int64_t k = 0; k < nRays; ++k) {
            const Frame<R>& fr = frames[rayList[3 * k]];
            RayTrace<R> rt;
            trace_ray(tris, tb.nodes, original, accel, rays != nullptr,
                      ray_origin(fr, rayList[3 * k + 1], rayList[3 * k + 2], nx, ny), fr.rayDir, maxBounces, dEdge,
                      dT, dDet, rt, cnt);
            queries += rt.queries;
            hitRays += rt.count > 0;
            bounces += (uint64_t)rt.count;
            if (rays) {
                oracle_ray& rr = rays[k];
                rr.count = rt.count;
                rr.amb = rt.amb;
                rr.dist = double(rt.dist);
                rr.normal[0] = rt.count ? double(rt.nLast.x) : 0.0;
                rr.normal[1] = rt.count ? double(rt.nLast.y) : 0.0;
                rr.normal[2] = rt.count ? double(rt.nLast.z) : 0.0;
                rr.lastdir[0] = rt.count ? double(rt.dLast.x) : 0.0;
                rr.lastdir[1] = rt.count ? double(rt.dLast.y) : 0.0;
                rr.lastdir[2] = rt.count ? double(rt.dLast.z) : 0.0;
                for (int q = 0; q < ORACLE_MAX_REC; ++q) rr.tri[q] = rt.ids[q];
            }
        }
        cHit += hitRays;
        cBounce += bounces;
        cQuery += queries;
        cBox += cnt.box;
        cTri += cnt.tri;
    }
    if (counts) {
        counts[0].rays = (uint64_t)nRays;
        counts[0].hit_rays = cHit;
        counts[0].bounces = cBounce;
        counts[0].queries = cQuery;
        counts[0].box_tests = cBox;
        counts[0].tri_tests = cTri;
    }
    return 0;
}

// Polarised variant (no counterpart in the reference, whose PO term is scalar):
// the same rays and hits in FP64, with the HH and VV incident fields tracked
// through every PEC reflection (E <- 2 (n.E) n - E) and, per exit ray that the
// scalar gate keeps (hit, cos(theta) = n.(-d_last) > 0), the co-polarised term
//   amplitude  2 R^n e.(n x (d_last x E_last))      (e = phi-hat for HH, theta-hat for VV)
//   path       dist + (s.llc - s.p_last)             (launch plane -> exit point -> plane)
//   term       k A / (4 pi) * amplitude * (-sin(k path), cos(k path)).
// Output: out[(a * nFreqs + f) * 2 + p] (p = 0 HH, 1 VV).
int sweep_pol_impl(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
                   const double* thetaDeg, const double* phiDeg, int64_t nAngles, const double* freqHz,
                   int64_t nFreqs, int32_t nx, int32_t ny, double gridSize, int32_t maxBounces, double reflConst,
                   int32_t accel, int32_t nThreads, double* outRe, double* outIm) {
    typedef double R;
    if (ntris <= 0 || nverts <= 0 || nx <= 0 || ny <= 0 || nAngles < 0 || nFreqs <= 0) return 1;
    std::vector<Tri<R>> tris(ntris);
    for (int64_t i = 0; i < ntris; ++i) {
        uint32_t a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        if (a >= nverts || b >= nverts || c >= nverts) return 2;
        auto P = [&](uint32_t k) {
            return V3<R>(R(xyz[3 * k]) * modelScale, R(xyz[3 * k + 1]) * modelScale, R(xyz[3 * k + 2]) * modelScale);
        };
        tris[i] = Tri<R>{P(a), P(b), P(c), (int32_t)i};
    }
    std::vector<Tri<R>> original = tris;
    TreeBuilder<R> tb(tris);
    if (accel == 1) tb.run();
#ifdef _OPENMP
    if (nThreads > 0) omp_set_num_threads(nThreads);
#endif
    const R G = gridSize;
    const R tMin = 0.001, tMax = 1e20, nudge = 1e-4;
    const R rayArea = (G * G) / R(int64_t(nx) * int64_t(ny));
    std::vector<R> kk(nFreqs);
    for (int64_t f = 0; f < nFreqs; ++f) kk[f] = 2.0 * M_PI / (299792458.0 / freqHz[f]);
    const size_t nc = (size_t)nFreqs * 2;
    std::vector<double> rowRe((size_t)ny * nc), rowIm((size_t)ny * nc);
    for (int64_t a = 0; a < nAngles; ++a) {
        Frame<R> fr = make_frame<R>(thetaDeg[a], phiDeg[a], G);
        const R th = thetaDeg[a] * M_PI / 180.0, ph = phiDeg[a] * M_PI / 180.0;
        const V3<R> eRx[2] = {V3<R>(-std::sin(ph), std::cos(ph), 0.0),
                              V3<R>(std::cos(th) * std::cos(ph), std::cos(th) * std::sin(ph), -std::sin(th))};
        const R plane = dot(fr.dir, fr.llc);
#pragma omp parallel for schedule(dynamic)
        for (int32_t j = 0; j < ny; ++j) {
            Counters cnt;
            std::vector<double> accRe(nc, 0.0), accIm(nc, 0.0);
            for (int32_t i = 0; i < nx; ++i) {
                R u = (R(i) + 0.5) / R(nx);
                R v = (R(j) + 0.5) / R(ny);
                V3<R> o = fr.llc + scale(u, fr.u) + scale(v, fr.v);
                V3<R> d = fr.rayDir;
                V3<R> E[2] = {eRx[0], eRx[1]};   // field on the current segment
                V3<R> Elast[2], nLast, dLast, pLast;
                int32_t count = 0;
                R dist = 0.0;
                for (int32_t b = 0; b < maxBounces; ++b) {
                    Hit<R> h;
                    bool hit = accel == 1 ? walk_tree(tris, tb.nodes, o, d, tMin, tMax, h, cnt)
                                          : walk_all(original, o, d, tMin, tMax, h, cnt);
                    if (!hit) break;
                    nLast = h.n;
                    dLast = d;
                    pLast = h.p;
                    count++;
                    dist += h.t;
                    for (int p = 0; p < 2; ++p) {
                        Elast[p] = E[p];
                        E[p] = scale(2.0 * dot(h.n, E[p]), h.n) - E[p];
                    }
                    d = unit(d - scale(R(2.0) * dot(d, h.n), h.n));
                    o = h.p + scale(nudge, h.n);
                }
                if (count == 0) continue;
                R Rn = 1.0;
                for (int32_t b = 0; b < count; ++b) Rn *= reflConst;
                if (!(dot(nLast, -dLast) > 0.0)) continue;
                const R path = dist + (plane - dot(fr.dir, pLast));
                R amp[2];
                for (int p = 0; p < 2; ++p) amp[p] = 2.0 * Rn * dot(eRx[p], cross(nLast, cross(dLast, Elast[p])));
                for (int64_t f = 0; f < nFreqs; ++f) {
                    const R k = kk[f];
                    const R phase = std::fmod(k * path, 2.0 * M_PI);
                    const R s = std::sin(phase), c = std::cos(phase);
                    for (int p = 0; p < 2; ++p) {
                        const R mag = (k * rayArea / (4.0 * M_PI)) * amp[p];
                        accRe[2 * f + p] += -mag * s;
                        accIm[2 * f + p] += mag * c;
                    }
                }
            }
            for (size_t c = 0; c < nc; ++c) {
                rowRe[(size_t)j * nc + c] = accRe[c];
                rowIm[(size_t)j * nc + c] = accIm[c];
            }
        }
        for (size_t c = 0; c < nc; ++c) {
            double re = 0, im = 0;
            for (int32_t j = 0; j < ny; ++j) { re += rowRe[(size_t)j * nc + c]; im += rowIm[(size_t)j * nc + c]; }
            outRe[(size_t)a * nc + c] = re;
            outIm[(size_t)a * nc + c] = im;
        }
    }
    return 0;
}

}  // namespace

extern "C" {

// Polarised FP64 sweep (see sweep_pol_impl); accel as oracle_sweep.
int oracle_sweep_pol(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
                     const double* thetaDeg, const double* phiDeg, int64_t nAngles, const double* freqHz,
                     int64_t nFreqs, int32_t nx, int32_t ny, double gridSize, int32_t maxBounces, double reflConst,
                     int32_t accel, int32_t nThreads, double* outRe, double* outIm) {
    return sweep_pol_impl(xyz, nverts, idx, ntris, modelScale, thetaDeg, phiDeg, nAngles, freqHz, nFreqs, nx, ny,
                          gridSize, maxBounces, reflConst, accel, nThreads, outRe, outIm);
}

// Full sweep: for every angle trace nx*ny rays (reference semantics) and reduce
// the PO field for every frequency.  precision: 64 or 32.  accel: 1 = reference
// SAH tree, 0 = brute force (with ambiguity flags when per-ray records are asked).
// Returns 0 on success.
int oracle_sweep(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
                 const double* thetaDeg, const double* phiDeg, int64_t nAngles, const double* freqHz,
                 int64_t nFreqs, int32_t nx, int32_t ny, double gridSize, int32_t maxBounces, double reflConst,
                 int32_t precision, int32_t accel, int32_t nThreads, double* outRe, double* outIm,
                 oracle_counts* counts, oracle_ray* rays, double dEdge, double dT, double dDet) {
    if (precision == 32)
        return sweep_impl<float>(xyz, nverts, idx, ntris, modelScale, thetaDeg, phiDeg, nAngles, freqHz, nFreqs, nx,
                                 ny, gridSize, maxBounces, reflConst, accel, nThreads, outRe, outIm, counts, rays,
                                 dEdge, dT, dDet);
    return sweep_impl<double>(xyz, nverts, idx, ntris, modelScale, thetaDeg, phiDeg, nAngles, freqHz, nFreqs, nx, ny,
                              gridSize, maxBounces, reflConst, accel, nThreads, outRe, outIm, counts, rays, dEdge, dT,
                              dDet);
}

// Traces an explicit list of rays (see trace_list_impl); precision 64 or 32, accel
// as oracle_sweep.  Returns 0 on success, 3 for a ray outside the angles or grid.
int oracle_trace_rays(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
                      const double* thetaDeg, const double* phiDeg, int64_t nAngles, const int32_t* rayList,
                      int64_t nRays, int32_t nx, int32_t ny, double gridSize, int32_t maxBounces, int32_t precision,
                      int32_t accel, int32_t nThreads, oracle_ray* rays, oracle_counts* counts, double dEdge,
                      double dT, double dDet) {
    if (precision == 32)
        return trace_list_impl<float>(xyz, nverts, idx, ntris, modelScale, thetaDeg, phiDeg, nAngles, rayList, nRays,
                                      nx, ny, gridSize, maxBounces, accel, nThreads, rays, counts, dEdge, dT, dDet);
    return trace_list_impl<double>(xyz, nverts, idx, ntris, modelScale, thetaDeg, phiDeg, nAngles, rayList, nRays, nx,
                                   ny, gridSize, maxBounces, accel, nThreads, rays, counts, dEdge, dT, dDet);
}

// Builds the reference SAH tree (FP64) and returns node count; when the output
// pointers are non-null they receive per node (lo.xyz, hi.xyz) and
// (left, right, first, count), and the triangle order (caller index per slot).
int64_t oracle_build_tree(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
                          double* nodeBounds, int32_t* nodeLinks, int32_t* triOrder) {
    std::vector<Tri<double>> tris(ntris);
    for (int64_t i = 0; i < ntris; ++i) {
        auto P = [&](uint32_t k) {
            return V3<double>(double(xyz[3 * k]) * modelScale, double(xyz[3 * k + 1]) * modelScale,
                              double(xyz[3 * k + 2]) * modelScale);
        };
        uint32_t a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        if (a >= nverts || b >= nverts || c >= nverts) return -1;
        tris[i] = Tri<double>{P(a), P(b), P(c), (int32_t)i};
    }
    TreeBuilder<double> tb(tris);
    tb.run();
    int64_t n = (int64_t)tb.nodes.size();
    for (int64_t k = 0; k < n && nodeBounds; ++k) {
        const auto& nd = tb.nodes[k];
        double* o = nodeBounds + 6 * k;
        o[0] = nd.lo.x; o[1] = nd.lo.y; o[2] = nd.lo.z; o[3] = nd.hi.x; o[4] = nd.hi.y; o[5] = nd.hi.z;
    }
    for (int64_t k = 0; k < n && nodeLinks; ++k) {
        const auto& nd = tb.nodes[k];
        int32_t* o = nodeLinks + 4 * k;
        o[0] = nd.left; o[1] = nd.right; o[2] = nd.first; o[3] = nd.count;
    }
    for (int64_t k = 0; k < ntris && triOrder; ++k) triOrder[k] = tris[k].id;
    return n;
}

// Launcher frame for one angle in FP64 (dir, u, v, llc as 12 doubles).
void oracle_frame(double thetaDeg, double phiDeg, double gridSize, double* out12) {
    Frame<double> f = make_frame<double>(thetaDeg, phiDeg, gridSize);
    double v[12] = {f.dir.x, f.dir.y, f.dir.z, f.u.x, f.u.y, f.u.z, f.v.x, f.v.y, f.v.z, f.llc.x, f.llc.y, f.llc.z};
    std::memcpy(out12, v, sizeof(v));
}

}  // extern "C"
