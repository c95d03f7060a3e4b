// cli.cpp -- RT-RCS: drop-in for the reference executable (src/RT-RCS.cpp,
// src/app/rtRcsEntry.cu:59-352) on top of libsbr.
//
//   RT-RCS --model m.obj|m.gltf|m.glb [freq] [--config c.txt] [--model-scale s]
//          [--freq-scan F_START F_END N]
//
// Reads config.txt (or --config), loads the model, builds the scene, runs the
// whole theta x phi sweep and writes rcs_results.csv in the working directory in
// the reference layout.  Exit status 1 on any error, with the reason on stderr.
// The sweep runs as one batched launch on the current GPU; the optional config
// keys `precision` (0 mixed, 1 FP32, 2 FP64) and `engine_mode` (0 batched, 1
// per-angle) select the other paths.  --freq-scan runs the reference's frequency
// scan in one process instead (results_freq_scans.csv).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
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

// Frequency scan (replaces util/run_freq_scan.sh:30-53, which re-runs RT-RCS per
// frequency and appends util/plotRCS.py's mean / sample standard deviation of
// rcs_m2 over the angle sweep to results_freq_scans.csv): the N frequencies
// round(logspace(F_START, F_END, N)) are traced as jobs of one plan on the
// config's grid -- at most 128 frequencies per job, all sharing each angle's trace.
int freq_scan(const sbr_config& cfg, sbr_scene* scene, double f0, double f1, int nf) {
    int64_t n = (int64_t)std::max(0, cfg.theta_samples) * std::max(0, cfg.phi_samples);
    std::vector<double> th(n), ph(n);
    sbr_config_angles(&cfg, th.data(), ph.data());
    std::vector<double> freqs(nf);
    for (int i = 0; i < nf; ++i) {
        const double e = nf > 1 ? std::log10(f0) + i * (std::log10(f1) - std::log10(f0)) / (nf - 1) : std::log10(f0);
        freqs[i] = std::round(std::pow(10.0, e));
    }
    std::vector<sbr_job> jobs;
    for (int k0 = 0; k0 < nf; k0 += 128)
        jobs.push_back(sbr_job{th.data(), ph.data(), n, freqs.data() + k0, std::min(128, nf - k0), cfg.nx, cfg.ny,
                               cfg.grid_size, cfg.max_bounces, cfg.reflection_const});
    // samples are (job, angle, frequency of the job)
    std::vector<double> sigma((size_t)n * nf);
    sbr_result res{};
    res.sigma_m2 = sigma.data();
    sbr_run_opts ro{};
    ro.mode = SBR_MODE_BATCHED;
    ro.precision = cfg.precision;
    sbr_status st = sbr_run(scene, jobs.data(), jobs.size(), &res, &ro);
    if (st != SBR_OK) return die("frequency scan", st);
    FILE* f = std::fopen("results_freq_scans.csv", "a");
    if (!f) {
        std::cerr << "Error: cannot write results_freq_scans.csv\n";
        return 1;
    }
    std::fseek(f, 0, SEEK_END);
    if (std::ftell(f) == 0) std::fprintf(f, "Frequency,Avg_RCS,Std_RCS\n");
    size_t base = 0;
    for (const sbr_job& J : jobs) {
        for (int64_t k = 0; k < J.n_freqs; ++k) {
            double s = 0.0, s2 = 0.0;
            for (int64_t a = 0; a < n; ++a) s += sigma[base + (size_t)a * J.n_freqs + k];
            const double mean = n > 0 ? s / double(n) : 0.0;
            for (int64_t a = 0; a < n; ++a) {
                const double d = sigma[base + (size_t)a * J.n_freqs + k] - mean;
                s2 += d * d;
            }
            const double sd = n > 1 ? std::sqrt(s2 / double(n - 1)) : 0.0;
            std::fprintf(f, "%.1f,%.17g,%.17g\n", J.freq_hz[k], mean, sd);
            std::cout << "Frequency " << J.freq_hz[k] << " Hz: average RCS " << mean << " +- " << sd << " m^2\n";
        }
        base += (size_t)n * J.n_freqs;
    }
    std::fclose(f);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    std::cerr << "SagittaSBR-compatible monostatic RCS (sbr-b200)\n";
    auto t0 = std::chrono::steady_clock::now();
    // --freq-scan F_START F_END N is this engine's own flag; the rest goes to loadConfig
    std::vector<const char*> args;
    double scan_f0 = 0.0, scan_f1 = 0.0;
    int scan_n = 0;
    for (int i = 0; i < argc; ++i) {
        if (std::string(argv[i]) == "--freq-scan") {
            if (i + 3 >= argc) {
                std::cerr << "Error: --freq-scan needs F_START F_END N\n";
                return 1;
            }
            scan_f0 = std::atof(argv[i + 1]);
            scan_f1 = std::atof(argv[i + 2]);
            scan_n = std::atoi(argv[i + 3]);
            if (!(scan_f0 > 0) || !(scan_f1 > 0) || scan_n < 1) {
                std::cerr << "Error: --freq-scan needs positive F_START, F_END and N >= 1\n";
                return 1;
            }
            i += 3;
            continue;
        }
        args.push_back(argv[i]);
    }
    sbr_config cfg;
    sbr_status st = sbr_config_load("config.txt", (int)args.size(), args.data(), &cfg);
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
    if (scan_n > 0) {
        const int rc = freq_scan(cfg, scene, scan_f0, scan_f1, scan_n);
        sbr_scene_destroy(scene);
        return rc;
    }

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
    std::vector<double> field(2 * n), err_db;
    res.field = field.data();
    res.sigma_m2 = sigma.data();
    res.rcs_dbsm = dbsm.data();
    res.stats = stats.data();
    st = sbr_run(scene, &job, 1, &res, &ro);
    if (st != SBR_OK) {
        sbr_scene_destroy(scene);
        return die("sweep", st);
    }
    // optional key error_bound: each row's stated bound against the FP64 result
    if (cfg.error_bound) {
        if (cfg.precision != SBR_PREC_MIXED) {
            std::cerr << "Warning: error_bound applies to mixed precision (precision 0); not stated.\n";
        } else {
            err_db.resize(n);
            st = sbr_error_bound(scene, &job, 1, &ro, field.data(), nullptr, err_db.data());
            if (st != SBR_OK) {
                sbr_scene_destroy(scene);
                return die("error bound", st);
            }
        }
    }
    st = sbr_write_csv_err("rcs_results.csv", &cfg, th.data(), ph.data(), sigma.data(), dbsm.data(),
                           err_db.empty() ? nullptr : err_db.data(), n);
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
