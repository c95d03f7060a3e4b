"""The host binned-SAH builder (sagittasbr_b200/csrc/bvh_build.cpp) on its own, on
the CPU: compiled with a small driver, run on seeded triangle boxes.

* every triangle lands in exactly one leaf, leaves hold 1..15 triangles;
* every node's box is the union of its children's (inner) or of its triangles'
  boxes (leaves) -- exact, as the traversal relies on conservative boxes;
* the tree does not depend on the thread count (subtrees built concurrently are
  renumbered in pre-order);
* a set of identical triangles (equal centroids) is split by the median fallback.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "sagittasbr_b200", "csrc")

DRIVER = r"""
#include "bvh_build.hpp"
#include <cstdio>
#include <cstdlib>
#include <vector>
using namespace sbr;
int main(int argc, char** argv) {
    const int threads = std::atoi(argv[3]), leaf = std::atoi(argv[4]);
    FILE* f = std::fopen(argv[1], "rb");
    std::fseek(f, 0, SEEK_END);
    const long nb = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<float> b(nb / 4);
    if (std::fread(b.data(), 4, b.size(), f) != b.size()) return 2;
    std::fclose(f);
    const size_t n = b.size() / 6;
    std::vector<float> lo(3 * n), hi(3 * n);
    for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) { lo[3 * i + a] = b[6 * i + a]; hi[3 * i + a] = b[6 * i + 3 + a]; }
    BuildOptions o;
    o.n_threads = threads;
    o.leaf_size = leaf;
    o.max_leaf = 15;
    BinTree t = build_sah(lo, hi, o);
    FILE* g = std::fopen(argv[2], "wb");
    const int32_t hdr[3] = {(int32_t)t.nodes.size(), (int32_t)t.order.size(), t.depth};
    std::fwrite(hdr, 4, 3, g);
    for (const BinNode& nd : t.nodes) std::fwrite(&nd, sizeof(BinNode), 1, g);
    std::fwrite(t.order.data(), 4, t.order.size(), g);
    std::fclose(g);
    return 0;
}
"""

NODE = np.dtype([("lo", "<f4", 3), ("hi", "<f4", 3), ("left", "<i4"), ("right", "<i4"), ("first", "<i4"),
                 ("count", "<i4")])


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("bvh")
    src = d / "driver.cpp"
    src.write_text(DRIVER)
    exe = d / "driver"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, "-I", "/usr/local/cuda/include",
                    str(src), os.path.join(CSRC, "bvh_build.cpp"), "-o", str(exe), "-lpthread"], check=True)
    return d, exe


def _build(driver, boxes, threads, leaf=3):
    d, exe = driver
    inp, out = d / "boxes.bin", d / f"tree_{threads}.bin"
    np.ascontiguousarray(boxes, dtype=np.float32).tofile(inp)
    subprocess.run([str(exe), str(inp), str(out), str(threads), str(leaf)], check=True)
    raw = np.fromfile(out, dtype=np.uint8)
    nn, no, depth = np.frombuffer(raw[:12], dtype="<i4")
    nodes = np.frombuffer(raw[12:12 + nn * NODE.itemsize], dtype=NODE)
    order = np.frombuffer(raw[12 + nn * NODE.itemsize:], dtype="<i4")
    assert order.size == no
    return nodes, order, int(depth)


def _boxes(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(n, 3)) * np.array([10.0, 2.0, 1.0])
    h = np.abs(rng.normal(size=(n, 3))) * 0.05
    return np.concatenate([c - h, c + h], axis=1).astype(np.float32)


def _check(nodes, order, boxes):
    n = boxes.shape[0]
    lo, hi = boxes[:, :3], boxes[:, 3:]
    seen = np.zeros(n, dtype=int)
    for k, nd in enumerate(nodes):
        if nd["left"] < 0:
            assert 1 <= nd["count"] <= 15
            tris = order[nd["first"]:nd["first"] + nd["count"]]
            seen[tris] += 1
            assert np.array_equal(nd["lo"], lo[tris].min(axis=0)) and np.array_equal(nd["hi"], hi[tris].max(axis=0))
        else:
            a, b = nodes[nd["left"]], nodes[nd["right"]]
            assert nd["left"] > k and nd["right"] > k  # pre-order
            assert np.array_equal(nd["lo"], np.minimum(a["lo"], b["lo"]))
            assert np.array_equal(nd["hi"], np.maximum(a["hi"], b["hi"]))
    assert np.all(seen == 1)


def test_tree_invariants_and_thread_independence(driver):
    boxes = _boxes(60000, 7)
    ref = None
    for threads in (1, 3, 8):
        nodes, order, depth = _build(driver, boxes, threads)
        _check(nodes, order, boxes)
        if ref is None:
            ref = (nodes.tobytes(), order.tobytes(), depth)
        else:
            assert (nodes.tobytes(), order.tobytes(), depth) == ref, threads


def test_equal_centroids_take_the_median_split(driver):
    one = np.array([[0.0, 0.0, 0.0, 1.0, 1.0, 1.0]], np.float32)
    boxes = np.concatenate([_boxes(200, 3), np.repeat(one, 40, axis=0)])
    nodes, order, _ = _build(driver, boxes, 1)
    _check(nodes, order, boxes)
    dup = set(range(200, 240))
    leaves = [set(order[nd["first"]:nd["first"] + nd["count"]]) for nd in nodes if nd["left"] < 0]
    holding = [lf & dup for lf in leaves if lf & dup]
    assert all(len(h) <= 15 for h in holding) and sum(len(h) for h in holding) == 40
