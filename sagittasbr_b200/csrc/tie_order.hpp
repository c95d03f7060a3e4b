// tie_order.hpp -- which of two triangles hit at exactly the same distance the
// reference's closest-hit walk keeps.
//
// The reference accepts a triangle whose hit distance equals the closest so far
// (`t > tMax` rejects, src/cuda/rtKernels.cu:36) and walks its binary tree in a
// fixed order (pop; inner node -> push left, then right, so the right subtree is
// visited first; leaf -> its triangles in order, src/cuda/rtKernels.cu:63-100).
// Node culling removes nodes but never reorders them, so among triangles hit at
// the same distance it keeps the one that comes last in that fixed order.  That
// order depends on its tree, built in its own arithmetic by binned SAH with
// std::partition and the std::nth_element median fallback
// (src/scene/bvhBuilder.cpp:93-312, leaves of 4, 16 bins).
//
// Exact ties decide results where a mesh holds the same triangle twice with
// opposite windings (two faces at one place, one of them facing the ray): the kept
// triangle's normal decides the PO term's obliquity test and the reflected ray.
// For such meshes the scene stores each triangle's rank in the reference's walk
// order, and the kernels keep, on an exact tie, the triangle of higher rank.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace sbr {

// True when two triangles have the same three vertex positions (bit for bit) with
// opposite windings.  Triangles with a repeated vertex are ignored.
bool has_opposed_twins(const float* xyz, const uint32_t* idx, size_t ntris);

// rank[t] = position of caller triangle t in the reference's walk order (0 first),
// for the tree the reference's FP64 build (USE_DOUBLE) makes of the vertices
// double(xyz) * scale.
std::vector<int32_t> reference_walk_rank(const float* xyz, const uint32_t* idx, size_t ntris, double scale,
                                         int n_threads);

}  // namespace sbr
