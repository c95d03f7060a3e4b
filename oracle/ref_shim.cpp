// ref_shim.cpp -- host driver around the reference's OWN code, compiled into
// oracle/_ref/ by oracle/Makefile from the sources where they lie (they are never
// copied into this repository).  Test infrastructure and CPU baseline only.
//
// Compiled pieces (by #include, resolved through the Makefile's -I paths):
//   src/cuda/rtKernels.cu      launchRaysMultiBounce + hitBvh/hitAabb/hitTriangle
//                              (run once per ray with blockIdx = (i, j))
//   src/scene/bvhBuilder.cpp   buildBvh (binned SAH), run with enableParallel=false
//                              so node numbering is deterministic.
// Restated here (the reference has them inside MPI/CUDA host code that cannot be
// compiled for the host): the launcher frame (src/app/sweep.cu:336-364), k and
// ray area (src/app/sweep.cu:50-55) and the PO term (src/cuda/poKernels.cu:81-109),
// summed in FP64 in ray order per row, rows in order.
//
// Build twice: with -DUSE_DOUBLE (the reference's FP64 build) and without (FP32).

#include "cuda_runtime.h"  // oracle/ref_include stand-in

thread_local ref_shim_dim3 blockIdx;
thread_local ref_shim_dim3 threadIdx;
thread_local ref_shim_dim3 blockDim;

#include "cuda/rtKernels.cu"
#include "scene/bvhBuilder.cpp"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct RefFrame {
    vec3 dir, rayDir, u, v, llc;
};

RefFrame ref_frame(double thetaDeg, double phiDeg, Real G) {
    Real th = Real(thetaDeg) * Real(M_PI) / REAL_CONST(180.0);
    Real ph = Real(phiDeg) * Real(M_PI) / REAL_CONST(180.0);
    RefFrame f;
    f.dir = vec3(std::sin(th) * std::cos(ph), std::sin(th) * std::sin(ph), std::cos(th));
    f.rayDir = -f.dir;
    vec3 up(0, 1, 0);
    if (std::fabs(f.dir.y()) > REAL_CONST(0.99)) up = vec3(1, 0, 0);
    f.u = unitVector(cross(up, f.dir)) * G;
    f.v = unitVector(cross(f.dir, f.u)) * G;
    f.llc = (f.dir * (REAL_CONST(10.0) * G)) - REAL_CONST(0.5) * f.u - REAL_CONST(0.5) * f.v;
    return f;
}

bvhBuildResult ref_tree(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
                        bool& ok) {
    std::vector<Triangle> tris;
    tris.reserve(ntris);
    const Real sc = Real(modelScale);
    ok = true;
    for (int64_t i = 0; i < ntris; ++i) {
        uint32_t a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        if (a >= nverts || b >= nverts || c >= nverts) { ok = false; return {}; }
        Triangle t;
        t.v0 = vec3(Real(xyz[3 * a]) * sc, Real(xyz[3 * a + 1]) * sc, Real(xyz[3 * a + 2]) * sc);
        t.v1 = vec3(Real(xyz[3 * b]) * sc, Real(xyz[3 * b + 1]) * sc, Real(xyz[3 * b + 2]) * sc);
        t.v2 = vec3(Real(xyz[3 * c]) * sc, Real(xyz[3 * c + 1]) * sc, Real(xyz[3 * c + 2]) * sc);
        tris.push_back(t);
    }
    bvhBuildOptions opts;
    opts.enableParallel = false;
    return buildBvh(std::move(tris), opts);
}

}  // namespace

extern "C" {

typedef struct ref_ray {
    int32_t count;
    int32_t pad;
    double dist;
    double normal[3];
    double lastdir[3];
} ref_ray;

int ref_real_bytes(void) { return (int)sizeof(Real); }

// Reference tree: node count; optional outputs as in oracle_build_tree, plus the
// reordered triangle vertices (9 doubles per slot).
int64_t ref_build_tree(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
                       double* nodeBounds, int32_t* nodeLinks, double* triVerts) {
    bool ok;
    bvhBuildResult r = ref_tree(xyz, nverts, idx, ntris, modelScale, ok);
    if (!ok) return -1;
    int64_t n = (int64_t)r.nodes.size();
    for (int64_t k = 0; k < n; ++k) {
        const BvhNode& nd = r.nodes[k];
        if (nodeBounds) {
            double* o = nodeBounds + 6 * k;
            o[0] = nd.boundsMin.x(); o[1] = nd.boundsMin.y(); o[2] = nd.boundsMin.z();
            o[3] = nd.boundsMax.x(); o[4] = nd.boundsMax.y(); o[5] = nd.boundsMax.z();
        }
        if (nodeLinks) {
            int32_t* o = nodeLinks + 4 * k;
            o[0] = nd.left; o[1] = nd.right; o[2] = nd.firstTri; o[3] = nd.triCount;
        }
    }
    for (int64_t k = 0; k < (int64_t)r.triangles.size() && triVerts; ++k) {
        const Triangle& t = r.triangles[k];
        double* o = triVerts + 9 * k;
        o[0] = t.v0.x(); o[1] = t.v0.y(); o[2] = t.v0.z();
        o[3] = t.v1.x(); o[4] = t.v1.y(); o[5] = t.v1.z();
        o[6] = t.v2.x(); o[7] = t.v2.y(); o[8] = t.v2.z();
    }
    return n;
}

// Sweep with the reference's per-ray routine on the host cores (OpenMP over ray
// rows).  Outputs the field per (angle, frequency); optional per-angle bounce sums
// and per-ray hit records.  Returns 0 on success.
int ref_sweep(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale,
              const double* thetaDeg, const double* phiDeg, int64_t nAngles, const double* freqHz, int64_t nFreqs,
              int32_t nx, int32_t ny, double gridSize, int32_t maxBounces, double reflConst, int32_t nThreads,
              double* outRe, double* outIm, uint64_t* bouncesPerAngle, ref_ray* rays) {
    if (ntris <= 0 || nx <= 0 || ny <= 0 || nFreqs <= 0) return 1;
    bool ok;
    bvhBuildResult tree = ref_tree(xyz, nverts, idx, ntris, modelScale, ok);
    if (!ok) return 2;
#ifdef _OPENMP
    if (nThreads > 0) omp_set_num_threads(nThreads);
#endif
    const Real G = Real(gridSize);
    const Real c0 = REAL_CONST(299792458.0);
    const Real rayArea = (G * G) / Real(int64_t(nx) * int64_t(ny));
    std::vector<Real> kk(nFreqs);
    for (int64_t f = 0; f < nFreqs; ++f) kk[f] = REAL_CONST(2.0) * Real(M_PI) / (c0 / Real(freqHz[f]));
    const size_t nRays = (size_t)nx * (size_t)ny;
    std::vector<vec3> hitNormal(nRays), lastDir(nRays);
    std::vector<Real> hitDist(nRays);
    std::vector<int> hitCount(nRays);
    std::vector<double> rowRe((size_t)ny * nFreqs), rowIm((size_t)ny * nFreqs);
    std::vector<uint64_t> rowB(ny);

    for (int64_t a = 0; a < nAngles; ++a) {
        RefFrame fr = ref_frame(thetaDeg[a], phiDeg[a], G);
#pragma omp parallel for schedule(dynamic)
        for (int32_t j = 0; j < ny; ++j) {
            blockDim = {1, 1, 1};
            threadIdx = {0, 0, 0};
            for (int32_t i = 0; i < nx; ++i) {
                blockIdx = {(unsigned)i, (unsigned)j, 0};
                launchRaysMultiBounce(hitNormal.data(), lastDir.data(), hitDist.data(), hitCount.data(), nx, ny,
                                      fr.llc, fr.u, fr.v, fr.rayDir, tree.triangles.data(), tree.nodes.data(),
                                      tree.rootIndex, maxBounces);
            }
            // PO term per ray (src/cuda/poKernels.cu:81-109), summed in FP64.
            uint64_t b = 0;
            for (int64_t f = 0; f < nFreqs; ++f) { rowRe[(size_t)j * nFreqs + f] = 0; rowIm[(size_t)j * nFreqs + f] = 0; }
            for (int32_t i = 0; i < nx; ++i) {
                size_t r = (size_t)j * nx + i;
                int n = hitCount[r];
                b += (uint64_t)n;
                if (n <= 0) continue;
                Real Rn = REAL_CONST(1.0);
                for (int q = 0; q < n; ++q) Rn *= Real(reflConst);
                Real cosT = dot(hitNormal[r], -lastDir[r]);
                if (!(cosT > REAL_CONST(0.0))) continue;
                for (int64_t f = 0; f < nFreqs; ++f) {
                    Real k = kk[f];
                    Real phase = REAL_CONST(2.0) * k * hitDist[r];
                    phase = std::fmod(phase, REAL_CONST(2.0) * Real(M_PI));
                    Real mag = (k * rayArea / (REAL_CONST(4.0) * Real(M_PI))) * REAL_CONST(2.0) * cosT * Rn;
                    rowRe[(size_t)j * nFreqs + f] += double(-mag * std::sin(phase));
                    rowIm[(size_t)j * nFreqs + f] += double(mag * std::cos(phase));
                }
            }
            rowB[j] = b;
        }
        uint64_t tb = 0;
        for (int64_t f = 0; f < nFreqs; ++f) {
            double re = 0, im = 0;
            for (int32_t j = 0; j < ny; ++j) { re += rowRe[(size_t)j * nFreqs + f]; im += rowIm[(size_t)j * nFreqs + f]; }
            outRe[a * nFreqs + f] = re;
            outIm[a * nFreqs + f] = im;
        }
        for (int32_t j = 0; j < ny; ++j) tb += rowB[j];
        if (bouncesPerAngle) bouncesPerAngle[a] = tb;
        if (rays) {
            for (size_t r = 0; r < nRays; ++r) {
                ref_ray& o = rays[(size_t)a * nRays + r];
                o.count = hitCount[r];
                o.pad = 0;
                o.dist = double(hitDist[r]);
                bool h = hitCount[r] > 0;
                o.normal[0] = h ? double(hitNormal[r].x()) : 0; o.normal[1] = h ? double(hitNormal[r].y()) : 0;
                o.normal[2] = h ? double(hitNormal[r].z()) : 0;
                o.lastdir[0] = h ? double(lastDir[r].x()) : 0; o.lastdir[1] = h ? double(lastDir[r].y()) : 0;
                o.lastdir[2] = h ? double(lastDir[r].z()) : 0;
            }
        }
    }
    return 0;
}


// ---- bounded samples of a sweep for the CPU baseline: the reference tree is built
// once per scene handle, then whole ray rows of chosen (angle, grid, frequency)
// samples are traced with the reference's own per-ray routine.

typedef struct ref_scene_h {
    bvhBuildResult tree;
} ref_scene_h;

void* ref_scene_create(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris, double modelScale) {
    bool ok;
    ref_scene_h* h = new ref_scene_h{ref_tree(xyz, nverts, idx, ntris, modelScale, ok)};
    if (!ok) {
        delete h;
        return nullptr;
    }
    return h;
}

void ref_scene_destroy(void* h) { delete static_cast<ref_scene_h*>(h); }

// Row k of the list is row j = rows[3k+2] of the n x n launcher (n = rows[3k+1]) of
// angle rows[3k], traced at frequency freqHz[k].  The routine is called with a one-row
// grid whose vertical edge is twice the row offset v V of the full grid, so its
// origins llc + u U + 0.5 (2 v V) equal the full grid's bit for bit without the
// nx*ny hit arrays of the full grid.  OpenMP over rows (dynamic); outRe/outIm get each
// row's PO sum (src/cuda/poKernels.cu:81-109) and *seconds the wall time of the
// traced rows (tree build excluded).  Returns 0 on success.
int ref_trace_rows(void* handle, const double* thetaDeg, const double* phiDeg, int64_t nAngles, const int32_t* rows,
                   int64_t nRows, const double* freqHz, double gridSize, int32_t maxBounces, double reflConst,
                   int32_t nThreads, double* outRe, double* outIm, uint64_t* raysOut, uint64_t* bouncesOut,
                   double* seconds) {
    ref_scene_h* h = static_cast<ref_scene_h*>(handle);
    if (!h || nRows < 0 || nAngles <= 0) return 1;
    int32_t nmax = 1;
    for (int64_t k = 0; k < nRows; ++k) {
        const int32_t a = rows[3 * k], n = rows[3 * k + 1], j = rows[3 * k + 2];
        if (a < 0 || a >= nAngles || n <= 0 || j < 0 || j >= n || !(freqHz[k] > 0)) return 3;
        nmax = std::max(nmax, n);
    }
#ifdef _OPENMP
    if (nThreads > 0) omp_set_num_threads(nThreads);
#endif
    const Real G = Real(gridSize);
    const Real c0 = REAL_CONST(299792458.0);
    uint64_t rays = 0, bounces = 0;
    const double t0 = omp_get_wtime();
#pragma omp parallel reduction(+ : rays, bounces)
    {
        std::vector<vec3> hitNormal(nmax), lastDir(nmax);
        std::vector<Real> hitDist(nmax);
        std::vector<int> hitCount(nmax);
        blockDim = {1, 1, 1};
        threadIdx = {0, 0, 0};
#pragma omp for schedule(dynamic)
        for (int64_t k = 0; k < nRows; ++k) {
            const int32_t a = rows[3 * k], n = rows[3 * k + 1], j = rows[3 * k + 2];
            RefFrame fr = ref_frame(thetaDeg[a], phiDeg[a], G);
            const Real v = (j + REAL_CONST(0.5)) / Real(n);
            const vec3 vert2 = (v * fr.v) * REAL_CONST(2.0);
            for (int32_t i = 0; i < n; ++i) {
                blockIdx = {(unsigned)i, 0u, 0u};
                launchRaysMultiBounce(hitNormal.data(), lastDir.data(), hitDist.data(), hitCount.data(), n, 1, fr.llc,
                                      fr.u, vert2, fr.rayDir, h->tree.triangles.data(), h->tree.nodes.data(),
                                      h->tree.rootIndex, maxBounces);
            }
            const Real kk = REAL_CONST(2.0) * Real(M_PI) / (c0 / Real(freqHz[k]));
            const Real rayArea = (G * G) / Real(int64_t(n) * int64_t(n));
            double re = 0, im = 0;
            for (int32_t i = 0; i < n; ++i) {
                const int cnt = hitCount[i];
                bounces += (uint64_t)cnt;
                if (cnt <= 0) continue;
                Real Rn = REAL_CONST(1.0);
                for (int q = 0; q < cnt; ++q) Rn *= Real(reflConst);
                Real cosT = dot(hitNormal[i], -lastDir[i]);
                if (!(cosT > REAL_CONST(0.0))) continue;
                Real phase = std::fmod(REAL_CONST(2.0) * kk * hitDist[i], REAL_CONST(2.0) * Real(M_PI));
                Real mag = (kk * rayArea / (REAL_CONST(4.0) * Real(M_PI))) * REAL_CONST(2.0) * cosT * Rn;
                re += double(-mag * std::sin(phase));
                im += double(mag * std::cos(phase));
            }
            rays += (uint64_t)n;
            if (outRe) outRe[k] = re;
            if (outIm) outIm[k] = im;
        }
    }
    if (seconds) *seconds = omp_get_wtime() - t0;
    if (raysOut) *raysOut = rays;
    if (bouncesOut) *bouncesOut = bounces;
    return 0;
}

}  // extern "C"
