// ref_gpu_shim.cu -- drives the reference's OWN GPU sweep (runSweep, src/app/sweep.cu,
// with launchRaysMultiBounce and integratePoMultiBounce from src/cuda/) on one GPU,
// compiled for sm_100a by baseline/Makefile from the sources where they lie (never
// copied into this repository).  This is the reference arm beside the engine's
// numbers: its per-angle FP32 (or -DUSE_DOUBLE) launch on the same B200.
//
// What this file adds around the reference code, following its own host set-up in
// runRcsApp (src/app/rtRcsEntry.cu:109-196): triangles scaled by modelScale in Real,
// buildBvh, device buffers for nx * ny rays, BVH upload, then one runSweep call per
// frequency.  The result rows runSweep writes (theta,phi,sigma,dBsm) are parsed back;
// the banner it prints to std::cerr is captured and the line "GPU Time (kernels only)"
// read from it.  The BVH is built serially (enableParallel = false) so that node
// numbering, and with it every run, is deterministic.

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "app/config.hpp"
#include "app/deviceBuffers.hpp"
#include "cuda/cudaUtils.cuh"
#include "scene/bvh.h"
#include "scene/bvhBuilder.hpp"
#include "sim/sweep.hpp"

#define SBRREF_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

double kernel_ms_from_banner(const std::string& banner) {
    const std::string key = "GPU Time (kernels only)";
    size_t at = banner.rfind(key);
    if (at == std::string::npos) return -1.0;
    at = banner.find(':', at + key.size());
    if (at == std::string::npos) return -1.0;
    return std::strtod(banner.c_str() + at + 1, nullptr);
}

}  // namespace

// Precision of the build: 32 (reference default) or 64 (-DUSE_DOUBLE).
SBRREF_EXPORT int sbrref_gpu_real_bits() { return int(sizeof(Real) * 8); }

// One reference sweep per frequency over the theta x phi grid
//   theta_t = th0 + t (th1 - th0) / (nth - 1),  phi_p = ph0 + p (ph1 - ph0) / (nph - 1)
// (the reference's own angle formula; one sample when n == 1).  Outputs, row-major in
// the reference's order (theta outer, phi inner): theta_out / phi_out [nth * nph] as the
// reference printed them, sigma_out [n_freqs][nth * nph] in m^2; per frequency the wall
// time of runSweep (s) and the reference's own summed RT + PO kernel time (ms).
// Returns 0, or -1 for bad arguments, -2 for an out-of-range index, -3 when the rows
// runSweep wrote cannot be read back.  A CUDA error inside the reference code ends the
// process (its checkCudaErrors calls exit(1)).
SBRREF_EXPORT int sbrref_gpu_sweep(const float* xyz, int64_t nverts, const uint32_t* idx, int64_t ntris,
                                   double model_scale, int n_freqs, const double* freqs, const int32_t* nx,
                                   const int32_t* ny, double grid_size, int max_bounces, double refl, double th0,
                                   double th1, int nth, double ph0, double ph1, int nph, double* theta_out,
                                   double* phi_out, double* sigma_out, double* wall_s_out, double* kernel_ms_out,
                                   double* build_s_out) {
    if (!xyz || !idx || nverts <= 0 || ntris <= 0 || n_freqs <= 0 || !freqs || !nx || !ny || nth <= 0 ||
        nph <= 0 || !sigma_out)
        return -1;
    std::vector<Triangle> tris;
    tris.reserve(size_t(ntris));
    const Real sc = Real(model_scale);
    for (int64_t i = 0; i < ntris; ++i) {
        const uint32_t a = idx[3 * i], b = idx[3 * i + 1], c = idx[3 * i + 2];
        if (int64_t(a) >= nverts || int64_t(b) >= nverts || int64_t(c) >= nverts) return -2;
        Triangle t;
        t.v0 = vec3(Real(xyz[3 * a]) * sc, Real(xyz[3 * a + 1]) * sc, Real(xyz[3 * a + 2]) * sc);
        t.v1 = vec3(Real(xyz[3 * b]) * sc, Real(xyz[3 * b + 1]) * sc, Real(xyz[3 * b + 2]) * sc);
        t.v2 = vec3(Real(xyz[3 * c]) * sc, Real(xyz[3 * c + 1]) * sc, Real(xyz[3 * c + 2]) * sc);
        tris.push_back(t);
    }
    int64_t max_rays = 0;
    for (int f = 0; f < n_freqs; ++f) {
        if (nx[f] <= 0 || ny[f] <= 0 || int64_t(nx[f]) * ny[f] > INT32_MAX) return -1;
        max_rays = std::max<int64_t>(max_rays, int64_t(nx[f]) * ny[f]);
    }

    auto tb = std::chrono::steady_clock::now();
    bvhBuildOptions opt;
    opt.enableParallel = false;
    bvhBuildResult bvh = buildBvh(std::move(tris), opt);
    if (build_s_out)
        *build_s_out = std::chrono::duration<double>(std::chrono::steady_clock::now() - tb).count();

    deviceBuffers buffers;
    allocateDeviceBuffers(buffers, int(max_rays));
    bvhGpuData bd;
    bd.triangleCount = int(bvh.triangles.size());
    bd.nodeCount = int(bvh.nodes.size());
    bd.rootIndex = bvh.rootIndex;
    checkCudaErrors(cudaMalloc(&bd.triangles, bd.triangleCount * sizeof(Triangle)));
    checkCudaErrors(cudaMemcpy(bd.triangles, bvh.triangles.data(), bd.triangleCount * sizeof(Triangle),
                               cudaMemcpyHostToDevice));
    checkCudaErrors(cudaMalloc(&bd.nodes, bd.nodeCount * sizeof(BvhNode)));
    checkCudaErrors(
        cudaMemcpy(bd.nodes, bvh.nodes.data(), bd.nodeCount * sizeof(BvhNode), cudaMemcpyHostToDevice));
    checkCudaErrors(cudaDeviceSynchronize());

    const int n_ang = nth * nph;
    int rc = 0;
    std::ostringstream banner;
    std::streambuf* saved_buf = std::cerr.rdbuf(banner.rdbuf());
    const std::ios::fmtflags saved_flags = std::cerr.flags();
    const std::streamsize saved_prec = std::cerr.precision();
    for (int f = 0; f < n_freqs && rc == 0; ++f) {
        simulationConfig cfg;
        cfg.thetaStart = Real(th0);
        cfg.thetaEnd = Real(th1);
        cfg.thetaSamples = nth;
        cfg.phiStart = Real(ph0);
        cfg.phiEnd = Real(ph1);
        cfg.phiSamples = nph;
        cfg.gridSize = Real(grid_size);
        cfg.nx = nx[f];
        cfg.ny = ny[f];
        cfg.maxBounces = max_bounces;
        cfg.reflectionConst = Real(refl);
        cfg.freq = Real(freqs[f]);
        cfg.showInfoGPU = false;
        cfg.showHitStats = false;
        cfg.modelScale = Real(model_scale);
        std::ostringstream rows;
        rows << std::setprecision(17);
        banner.str("");
        checkCudaErrors(cudaDeviceSynchronize());
        auto t0 = std::chrono::steady_clock::now();
        runSweep(cfg, buffers, bd, rows);
        checkCudaErrors(cudaDeviceSynchronize());
        if (wall_s_out)
            wall_s_out[f] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (kernel_ms_out) kernel_ms_out[f] = kernel_ms_from_banner(banner.str());
        std::istringstream in(rows.str());
        std::string line;
        int k = 0;
        while (std::getline(in, line) && k < n_ang) {
            double th, ph, sg, db;
            if (std::sscanf(line.c_str(), "%lf,%lf,%lf,%lf", &th, &ph, &sg, &db) != 4) break;
            if (f == 0 && theta_out) theta_out[k] = th;
            if (f == 0 && phi_out) phi_out[k] = ph;
            sigma_out[int64_t(f) * n_ang + k] = sg;
            ++k;
        }
        if (k != n_ang) rc = -3;
    }
    std::cerr.rdbuf(saved_buf);
    std::cerr.flags(saved_flags);
    std::cerr.precision(saved_prec);

    checkCudaErrors(cudaFree(bd.triangles));
    checkCudaErrors(cudaFree(bd.nodes));
    freeDeviceBuffers(buffers);
    return rc;
}
