// ref_loader_shim.cpp -- the reference's OWN model loader (src/modelLoader.cpp with
// its vendored tinyobjloader / tinygltf), compiled for the host into oracle/_ref by
// oracle/Makefile from the sources where they lie, behind one C entry point that
// also de-indexes the mesh with the model scale as runRcsApp does
// (src/app/rtRcsEntry.cu:108-145, the FP32 build: float(position) * float(scale)).
// Test infrastructure only: it pins sbr_load_model's triangles to the reference's.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>

#include "modelLoader.hpp"

extern "C" {

// Loads `path` with modelLoader::loadModel and writes the de-indexed triangles
// (9 floats each: v0, v1, v2) to a malloc'd array.  Returns 0 on success, 1 when the
// loader fails, 2 for an empty or malformed index list, 3 for an out-of-range index;
// `err` receives the loader's message.
int ref_load_triangles(const char* path, double modelScale, float** out, size_t* ntris, char* err, size_t errlen) {
    modelLoader::MeshData mesh;
    std::string msg;
    *out = nullptr;
    *ntris = 0;
    auto put = [&](const std::string& m) {
        if (err && errlen) {
            std::strncpy(err, m.c_str(), errlen - 1);
            err[errlen - 1] = 0;
        }
    };
    if (!modelLoader::loadModel(path, mesh, msg)) {
        put(msg);
        return 1;
    }
    put(msg);
    if (mesh.indices.empty() || mesh.positions.empty() || mesh.indices.size() % 3 != 0) return 2;
    const size_t nv = mesh.positions.size() / 3, nt = mesh.indices.size() / 3;
    float* o = static_cast<float*>(std::malloc(nt * 9 * sizeof(float)));
    const float sc = float(modelScale);
    for (size_t t = 0; t < nt; ++t) {
        for (int c = 0; c < 3; ++c) {
            const uint32_t i = mesh.indices[3 * t + c];
            if (i >= nv) {
                std::free(o);
                return 3;
            }
            for (int k = 0; k < 3; ++k) o[9 * t + 3 * c + k] = mesh.positions[3 * i + k] * sc;
        }
    }
    *out = o;
    *ntris = nt;
    return 0;
}

void ref_free(void* p) { std::free(p); }

}  // extern "C"
