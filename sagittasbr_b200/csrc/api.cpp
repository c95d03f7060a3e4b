// api.cpp -- status strings, error detail, and the reference's entry surface:
// config.txt / command line (src/app/config.cpp:11-155), the theta-major angle
// grid (src/app/sweep.cu:336-347), OBJ input and the rcs_results.csv layout
// (src/app/rtRcsEntry.cu:298-303, src/app/sweep.cu:540-544).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "common.hpp"

namespace sbr {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

sbr_status fail(sbr_status s, const std::string& msg) {
    set_error(msg);
    return s;
}

sbr_status cuda_fail(cudaError_t e, const char* what) {
    set_error(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    if (e == cudaErrorMemoryAllocation) return SBR_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return SBR_ERR_NO_DEVICE;
    return SBR_ERR_CUDA;
}

}  // namespace sbr

using sbr::fail;

extern "C" {

const char* sbr_status_str(sbr_status s) {
    switch (s) {
        case SBR_OK: return "SBR_OK";
        case SBR_ERR_INVALID_ARG: return "SBR_ERR_INVALID_ARG";
        case SBR_ERR_EMPTY_MESH: return "SBR_ERR_EMPTY_MESH";
        case SBR_ERR_BAD_INDEX: return "SBR_ERR_BAD_INDEX";
        case SBR_ERR_NONFINITE: return "SBR_ERR_NONFINITE";
        case SBR_ERR_TOO_LARGE: return "SBR_ERR_TOO_LARGE";
        case SBR_ERR_CUDA: return "SBR_ERR_CUDA";
        case SBR_ERR_OOM: return "SBR_ERR_OOM";
        case SBR_ERR_NO_DEVICE: return "SBR_ERR_NO_DEVICE";
        case SBR_ERR_STACK: return "SBR_ERR_STACK";
        case SBR_ERR_TIMEOUT: return "SBR_ERR_TIMEOUT";
        case SBR_ERR_CANCELLED: return "SBR_ERR_CANCELLED";
        case SBR_ERR_IO: return "SBR_ERR_IO";
        case SBR_ERR_PARSE: return "SBR_ERR_PARSE";
        case SBR_ERR_UNSUPPORTED: return "SBR_ERR_UNSUPPORTED";
        default: return "SBR_ERR_UNKNOWN";
    }
}

const char* sbr_last_error(void) { return sbr::g_last_error.c_str(); }

int32_t sbr_abi_version(void) { return SBR_ABI_VERSION; }

void sbr_free(void* p) { std::free(p); }

// ------------------------------------------------------------------ config
sbr_status sbr_config_load(const char* default_path, int argc, const char* const* argv, sbr_config* out) {
    if (!out) return fail(SBR_ERR_INVALID_ARG, "out is null");
    sbr_config c{};
    c.phi_start = 0.0;
    c.phi_end = 180.0;
    c.phi_samples = 181;
    c.theta_start = 90.0;
    c.theta_end = 90.0;
    c.theta_samples = 1;
    c.grid_size = 10.0;
    c.nx = 5000;
    c.ny = 5000;
    c.tpb_x = 16;
    c.tpb_y = 16;
    c.max_bounces = 20;
    c.reflection_const = 1.0;
    c.freq = 10.0e9;
    c.show_info_gpu = 1;
    c.show_hit_stats = 1;
    c.model_scale = 1.0;
    c.model_path[0] = '\0';
    c.freq_source = 0;

    std::string path = default_path ? default_path : "config.txt";
    for (int i = 1; i < argc; ++i) {
        if (std::strcmp(argv[i], "--config") == 0 && i + 1 < argc) {
            path = argv[i + 1];
            break;
        }
    }
    // key value lines; '#' starts a comment; values read as double
    std::map<std::string, double> kv;
    std::ifstream in(path);
    if (!in.is_open()) {
        std::cerr << "Warning: Could not open " << path << ". Using defaults." << std::endl;
    } else {
        std::string line;
        while (std::getline(in, line)) {
            size_t h = line.find('#');
            if (h != std::string::npos) line.resize(h);
            std::istringstream ls(line);
            std::string key;
            double val;
            if (ls >> key >> val) kv[key] = val;
        }
    }
    auto has = [&](const char* k) { return kv.count(k) != 0; };
    if (has("phi_start")) c.phi_start = kv["phi_start"];
    if (has("phi_end")) c.phi_end = kv["phi_end"];
    if (has("phi_samples")) c.phi_samples = (int32_t)kv["phi_samples"];
    if (has("theta_start")) c.theta_start = kv["theta_start"];
    if (has("theta_end")) c.theta_end = kv["theta_end"];
    if (has("theta_samples")) c.theta_samples = (int32_t)kv["theta_samples"];
    if (has("grid_size")) c.grid_size = kv["grid_size"];
    if (has("n_x")) c.nx = (int32_t)kv["n_x"];
    if (has("n_y")) c.ny = (int32_t)kv["n_y"];
    if (has("tpb_x")) c.tpb_x = (int32_t)kv["tpb_x"];
    if (has("tpb_y")) c.tpb_y = (int32_t)kv["tpb_y"];
    if (has("max_bounces")) c.max_bounces = (int32_t)kv["max_bounces"];
    if (has("reflection_const")) c.reflection_const = kv["reflection_const"];
    if (has("show_info_GPU")) c.show_info_gpu = kv["show_info_GPU"] != 0.0;
    if (has("show_hit_stats")) c.show_hit_stats = kv["show_hit_stats"] != 0.0;
    if (has("freq")) {
        c.freq = kv["freq"];
        c.freq_source = 1;
    }
    c.precision = SBR_PREC_MIXED;
    c.mode = SBR_MODE_BATCHED;
    if (has("precision")) c.precision = (int32_t)kv["precision"];
    if (has("engine_mode")) c.mode = (int32_t)kv["engine_mode"];
    if (has("csv_digits")) c.csv_digits = (int32_t)kv["csv_digits"];
    if (has("error_bound")) c.error_bound = kv["error_bound"] != 0.0;

    bool freqCli = false;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--model") {
            if (i + 1 >= argc) return fail(SBR_ERR_INVALID_ARG, "Error: --model requires a file path.");
            std::snprintf(c.model_path, sizeof(c.model_path), "%s", argv[++i]);
            continue;
        }
        if (a == "--model-scale") {
            if (i + 1 >= argc) return fail(SBR_ERR_INVALID_ARG, "Error: --model-scale requires a numeric value.");
            c.model_scale = std::atof(argv[++i]);
            continue;
        }
        if (a == "--config") {
            ++i;
            continue;
        }
        if (a == "--full-precision") {
            c.csv_digits = 17;
            continue;
        }
        if (!a.empty() && a[0] != '-') {
            if (!freqCli) {
                c.freq = std::atof(a.c_str());
                freqCli = true;
                c.freq_source = 2;
            }
            continue;
        }
        std::cerr << "Warning: Unrecognized argument '" << a << "'.\n";
    }
    *out = c;
    return SBR_OK;
}

sbr_status sbr_config_angles(const sbr_config* c, double* theta, double* phi) {
    if (!c || !theta || !phi) return fail(SBR_ERR_INVALID_ARG, "null argument");
    if (c->theta_samples < 0 || c->phi_samples < 0) return fail(SBR_ERR_INVALID_ARG, "negative sample count");
    int64_t n = 0;
    for (int t = 0; t < c->theta_samples; ++t) {
        double th = c->theta_start +
                    (c->theta_samples > 1 ? t * (c->theta_end - c->theta_start) / (c->theta_samples - 1) : 0);
        for (int p = 0; p < c->phi_samples; ++p) {
            double ph = c->phi_start + (c->phi_samples > 1 ? p * (c->phi_end - c->phi_start) / (c->phi_samples - 1) : 0);
            theta[n] = th;
            phi[n] = ph;
            ++n;
        }
    }
    return SBR_OK;
}

// --------------------------------------------------------------------- OBJ
// v / f records.  Face tokens are v, v/vt, v//vn or v/vt/vn with 1-based or
// negative (relative) indices.  Quads are split along the shorter diagonal, as
// the vendored tinyobjloader used by the reference does with triangulate=true;
// larger polygons are fan-triangulated.
sbr_status sbr_load_obj(const char* path, float** xyz, size_t* nverts, uint32_t** tri_idx, size_t* ntris) {
    if (!path || !xyz || !nverts || !tri_idx || !ntris) return fail(SBR_ERR_INVALID_ARG, "null argument");
    *xyz = nullptr;
    *tri_idx = nullptr;
    *nverts = *ntris = 0;
    std::ifstream in(path);
    if (!in.is_open()) return fail(SBR_ERR_IO, std::string("cannot open ") + path);
    std::vector<float> V;
    std::vector<uint32_t> T;
    std::string line;
    size_t lineNo = 0;
    while (std::getline(in, line)) {
        ++lineNo;
        size_t b = line.find_first_not_of(" \t\r");
        if (b == std::string::npos || line[b] == '#') continue;
        if (line.compare(b, 2, "v ") == 0 || line.compare(b, 2, "v\t") == 0) {
            std::istringstream ls(line.substr(b + 2));
            double x, y, z;
            if (!(ls >> x >> y >> z)) return fail(SBR_ERR_PARSE, "bad vertex on line " + std::to_string(lineNo));
            V.push_back(float(x));
            V.push_back(float(y));
            V.push_back(float(z));
        } else if (line.compare(b, 2, "f ") == 0 || line.compare(b, 2, "f\t") == 0) {
            std::istringstream ls(line.substr(b + 2));
            std::string tok;
            std::vector<int64_t> face;
            int64_t nv = (int64_t)(V.size() / 3);
            while (ls >> tok) {
                size_t s = tok.find('/');
                long long k = std::atoll(tok.substr(0, s).c_str());
                if (k == 0) return fail(SBR_ERR_PARSE, "bad face index on line " + std::to_string(lineNo));
                int64_t ix = k > 0 ? k - 1 : nv + k;
                if (ix < 0 || ix >= nv) return fail(SBR_ERR_BAD_INDEX, "face index out of range on line " + std::to_string(lineNo));
                face.push_back(ix);
            }
            if (face.size() < 3) continue;
            if (face.size() == 4) {
                // squared diagonal lengths in FP32, summed x, y, z in order, as the
                // loader computes them (real_t = float; near-square quads depend on it)
                auto d2 = [&](int64_t a, int64_t c) {
                    const float dx = V[3 * c] - V[3 * a], dy = V[3 * c + 1] - V[3 * a + 1],
                                dz = V[3 * c + 2] - V[3 * a + 2];
                    return dx * dx + dy * dy + dz * dz;
                };
                if (d2(face[0], face[2]) < d2(face[1], face[3])) {
                    uint32_t t6[6] = {(uint32_t)face[0], (uint32_t)face[1], (uint32_t)face[2],
                                      (uint32_t)face[0], (uint32_t)face[2], (uint32_t)face[3]};
                    T.insert(T.end(), t6, t6 + 6);
                } else {
                    uint32_t t6[6] = {(uint32_t)face[0], (uint32_t)face[1], (uint32_t)face[3],
                                      (uint32_t)face[1], (uint32_t)face[2], (uint32_t)face[3]};
                    T.insert(T.end(), t6, t6 + 6);
                }
            } else {
                for (size_t q = 1; q + 1 < face.size(); ++q) {
                    T.push_back((uint32_t)face[0]);
                    T.push_back((uint32_t)face[q]);
                    T.push_back((uint32_t)face[q + 1]);
                }
            }
        }
    }
    if (T.empty()) return fail(SBR_ERR_EMPTY_MESH, std::string("no triangles in ") + path);
    *xyz = (float*)std::malloc(V.size() * sizeof(float));
    *tri_idx = (uint32_t*)std::malloc(T.size() * sizeof(uint32_t));
    if (!*xyz || !*tri_idx) {
        std::free(*xyz);
        std::free(*tri_idx);
        *xyz = nullptr;
        *tri_idx = nullptr;
        return fail(SBR_ERR_OOM, "host allocation failed");
    }
    std::memcpy(*xyz, V.data(), V.size() * sizeof(float));
    std::memcpy(*tri_idx, T.data(), T.size() * sizeof(uint32_t));
    *nverts = V.size() / 3;
    *ntris = T.size() / 3;
    return SBR_OK;
}

// --------------------------------------------------------------------- CSV
sbr_status sbr_write_csv(const char* path, const sbr_config* c, const double* theta, const double* phi,
                         const double* sigma, const double* dbsm, int64_t n) {
    return sbr_write_csv_err(path, c, theta, phi, sigma, dbsm, nullptr, n);
}

sbr_status sbr_write_csv_err(const char* path, const sbr_config* c, const double* theta, const double* phi,
                             const double* sigma, const double* dbsm, const double* err_db, int64_t n) {
    if (!path || !c || (n > 0 && (!theta || !phi || !sigma || !dbsm))) return fail(SBR_ERR_INVALID_ARG, "null argument");
    if (c->csv_digits < 0 || c->csv_digits > 17) return fail(SBR_ERR_INVALID_ARG, "csv_digits must be 0..17");
    std::ofstream f(path);
    if (!f.is_open()) return fail(SBR_ERR_IO, std::string("cannot write ") + path);
    // default ostream formatting (6 significant digits), as the reference's
    f << "# Frequency: " << c->freq << "\n# Grid: " << c->nx << "x" << c->ny << "\n";
    f << "# GridSize: " << c->grid_size << "\n# ThetaSamples: " << c->theta_samples << "\n";
    f << "# PhiSamples: " << c->phi_samples << "\n"
      << (err_db ? "theta,phi,rcs_m2,rcs_dbsm,rcs_err_db\n" : "theta,phi,rcs_m2,rcs_dbsm\n");
    if (c->csv_digits > 0) f << std::setprecision(c->csv_digits);
    for (int64_t i = 0; i < n; ++i) {
        f << theta[i] << "," << phi[i] << "," << sigma[i] << "," << dbsm[i];
        if (err_db) f << "," << err_db[i];
        f << "\n";
    }
    if (!f.good()) return fail(SBR_ERR_IO, std::string("write failed: ") + path);
    return SBR_OK;
}

}  // extern "C"
