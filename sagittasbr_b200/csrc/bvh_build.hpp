// bvh_build.hpp -- host binned-SAH BVH builder (deterministic output, parallel
// over subtrees) and its conversion to the GPU node layout.
//
// Same family as the reference builder (src/scene/bvhBuilder.cpp:115-312: binned
// SAH over centroids on all three axes, 16 bins, leaves of up to 4 triangles,
// median fallback) but written for this engine: bins are filled from per-triangle
// boxes computed once, the partition is by bin index so binning and splitting
// agree exactly, subtrees above a size threshold are built on separate threads,
// and the tree is renumbered in pre-order at the end so the node order does not
// depend on thread timing (the reference's atomic counter does,
// src/scene/bvhBuilder.cpp:245-248).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace sbr {

struct BuildOptions {
    int leaf_size = 4;     // split while more triangles than this
    int bin_count = 16;
    int n_threads = 0;     // 0 -> hardware concurrency
    int max_leaf = 15;     // hard cap (GPU leaf encoding)
};

struct BinNode {
    float lo[3], hi[3];
    int32_t left, right;   // child indices (-1 for leaves)
    int32_t first, count;  // triangle range in the permuted order (leaves)
};

struct BinTree {
    std::vector<BinNode> nodes;      // pre-order, root = 0
    std::vector<int32_t> order;      // slot -> caller triangle index
    int depth = 0;
};

// tri_lo/tri_hi: per-triangle boxes (3 floats each), used for the build.
BinTree build_sah(const std::vector<float>& tri_lo, const std::vector<float>& tri_hi, const BuildOptions& opt);

// The same tree built on the current CUDA device (gpu_build.cu): identical nodes,
// boxes and leaf triangle sets; triangles inside a leaf may be in another order.
// Returns false with the CUDA error in *err when a CUDA call fails.
bool build_sah_gpu(const std::vector<float>& tri_lo, const std::vector<float>& tri_hi, const BuildOptions& opt,
                   cudaStream_t stream, BinTree& out, cudaError_t* err);

}  // namespace sbr
