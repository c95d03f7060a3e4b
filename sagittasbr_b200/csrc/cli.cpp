// cli.cpp -- RT-RCS: drop-in for the reference executable (src/RT-RCS.cpp,
// src/app/rtRcsEntry.cu:59-352) on top of libsbr.
//
//   RT-RCS --model m.obj [freq] [--config c.txt] [--model-scale s]
//
// Reads config.txt (or --config), loads the OBJ model, builds the scene, runs the
// whole theta x phi sweep and writes rcs_results.csv in the working directory in
// the reference layout.  Exit status 1 on any error, with the reason on stderr.
// The sweep runs as one batched launch on the current GPU; the optional config
// keys `precision` (0 mixed, 1 FP32, 2 FP64) and `engine_mode` (0 batched, 1
// per-angle) select the other paths.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "sbr.h"

namespace {

bool ends_with(std::string s, const std::string& suf) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

int die(const char* what, sbr_status st) {
    std::cerr << "Error: " << what << ": " << sbr_status_str(st) << " (" << sbr_last_error() << ")\n";
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    std::cerr << "SagittaSBR-compatible monostatic RCS (sbr-b200)\n";
    auto t0 = std::chrono::steady_clock::now();
    sbr_config cfg;
    sbr_status st = sbr_config_load("config.txt", argc, (const char* const*)argv, &cfg);
    if (st != SBR_OK) {
        std::cerr << sbr_last_error() << "\n";
        return 1;
    }
    if (cfg.freq_source == 2) std::cout << "Using frequency from command line: " << cfg.freq << " Hz\n";
    else if (cfg.freq_source == 1) std::cout << "Using frequency from config file: " << cfg.freq << " Hz\n";
    else std::cout << "Using default frequency: " << cfg.freq << " Hz\n";
    std::string model = cfg.model_path;
    if (model.empty()) {
        std::cerr << "Error: --model is required for simulation runs.\n";
        return 1;
    }
    if (!ends_with(model, ".obj") && !ends_with(model, ".gltf") && !ends_with(model, ".glb")) {
        std::cerr << "Error: Unsupported model extension for '" << model << "'.\n";
        return 1;
    }
    float* xyz = nullptr;
    uint32_t* idx = nullptr;
    size_t nv = 0, nt = 0;
    st = sbr_load_model(model.c_str(), &xyz, &nv, &idx, &nt);
    if (st != SBR_OK) {
        std::cerr << "Error: Failed to load model '" << model << "'.\n" << sbr_last_error() << "\n";
        return 1;
    }
    sbr_build_opts bo{};
    bo.model_scale = cfg.model_scale;
    bo.device = -1;
    sbr_scene* scene = nullptr;
    st = sbr_scene_create(xyz, nv, idx, nt, &bo, &scene);
    sbr_free(xyz);
    sbr_free(idx);
    if (st != SBR_OK) return die("scene", st);
    sbr_scene_info si;
    sbr_scene_info_get(scene, &si);

    int64_t n = (int64_t)std::max(0, cfg.theta_samples) * std::max(0, cfg.phi_samples);
    std::vector<double> th(n), ph(n), sigma(n), dbsm(n);
    std::vector<uint64_t> stats(4 * n);
    sbr_config_angles(&cfg, th.data(), ph.data());
    double freq = cfg.freq;
    sbr_job job{th.data(), ph.data(), n, &freq, 1, cfg.nx, cfg.ny, cfg.grid_size, cfg.max_bounces, cfg.reflection_const};
    sbr_run_opts ro{};
    ro.mode = cfg.mode;
    ro.precision = cfg.precision;
    sbr_result res{};
    res.sigma_m2 = sigma.data();
    res.rcs_dbsm = dbsm.data();
    res.stats = stats.data();
    st = sbr_run(scene, &job, 1, &res, &ro);
    if (st != SBR_OK) {
        sbr_scene_destroy(scene);
        return die("sweep", st);
    }
    st = sbr_write_csv("rcs_results.csv", &cfg, th.data(), ph.data(), sigma.data(), dbsm.data(), n);
    if (st != SBR_OK) {
        sbr_scene_destroy(scene);
        return die("csv", st);
    }
    // per-angle hit statistics (src/app/sweep.cu:257-295): the hit fraction of the
    // full nx x ny grid and the mean hit count of the rays that hit, from the
    // counters the kernel keeps on the device (no per-ray copy to the host)
    if (cfg.show_hit_stats) {
        const double grid = double(cfg.nx) * double(cfg.ny);
        for (int64_t i = 0; i < n; ++i) {
            const double h = double(stats[4 * i + 1]), b = double(stats[4 * i + 2]);
            std::cerr << "[R0:" << std::setw(3) << i + 1 << "/" << n << "]"
                      << " | Theta: " << std::setw(3) << static_cast<int>(th[i]) << " deg"
                      << " | Phi: " << std::setw(3) << static_cast<int>(ph[i]) << " deg"
                      << " | Hit: " << std::fixed << std::setprecision(0) << 100.0 * h / grid << "%"
                      << " | Bounces: " << std::setprecision(2) << (h > 0 ? b / h : 0.0) << "\n";
        }
        std::cerr.unsetf(std::ios::floatfield);
        std::cerr << std::setprecision(6);
    }
    uint64_t rays = 0, hit = 0, bounces = 0, queries = 0;
    for (int64_t i = 0; i < n; ++i) {
        rays += stats[4 * i];
        hit += stats[4 * i + 1];
        bounces += stats[4 * i + 2];
        queries += stats[4 * i + 3];
    }
    double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::cerr << "Triangles           : " << si.n_triangles << "\n"
              << "BVH build           : " << si.build_ms << " ms (depth " << si.bvh_depth << ")\n"
              << "Angles              : " << n << "\n"
              << "Rays launched       : " << rays << " (grid " << (int64_t)cfg.nx * cfg.ny * n << ")\n"
              << "Hit rays            : " << hit << "\n"
              << "Bounces             : " << bounces << "\n"
              << "Closest-hit queries : " << queries << "\n"
              << "Sweep device time   : " << res.device_ms << " ms\n"
              << "Total wall time     : " << wall << " ms\n";
    sbr_scene_destroy(scene);
    return 0;
}
