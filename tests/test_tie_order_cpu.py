"""The exact-tie order (sagittasbr_b200/csrc/tie_order.cpp) on the CPU: compiled with
a small driver, run on meshes with and without coincident faces.

The reference keeps, among triangles hit at exactly the same distance, the one its
walk tests last (src/cuda/rtKernels.cu:36,63-100), so the engine stores each
triangle's rank in that walk where a mesh holds a triangle twice with opposite
windings.  Checked here:

* the rank order equals the walk order over the oracle's restated reference tree
  (src/scene/bvhBuilder.cpp, pinned to the reference's own builder by
  test_oracle.py), with the thread count not mattering;
* where the reference tree is present, it equals the walk order over the tree the
  reference's own FP64 builder makes (oracle/_ref), on every OBJ model it ships;
* twins are found for opposite windings only (same-winding copies and triangles
  with a repeated vertex do not count).
"""
import os
import subprocess

import numpy as np
import pytest

from sagittasbr_b200 import meshes as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "sagittasbr_b200", "csrc")

DRIVER = r"""
#include "tie_order.hpp"
#include <cstdio>
#include <cstdlib>
#include <vector>
int main(int argc, char** argv) {
    FILE* f = std::fopen(argv[1], "rb");
    long long nv, nt;
    if (std::fread(&nv, 8, 1, f) != 1 || std::fread(&nt, 8, 1, f) != 1) return 2;
    std::vector<float> xyz(3 * nv);
    std::vector<uint32_t> idx(3 * nt);
    if (std::fread(xyz.data(), 4, xyz.size(), f) != xyz.size()) return 3;
    if (std::fread(idx.data(), 4, idx.size(), f) != idx.size()) return 3;
    std::fclose(f);
    const int twins = sbr::has_opposed_twins(xyz.data(), idx.data(), nt) ? 1 : 0;
    std::vector<int32_t> r = sbr::reference_walk_rank(xyz.data(), idx.data(), nt, std::atof(argv[3]),
                                                      std::atoi(argv[4]));
    FILE* g = std::fopen(argv[2], "wb");
    std::fwrite(&twins, 4, 1, g);
    std::fwrite(r.data(), 4, r.size(), g);
    std::fclose(g);
    return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("tie")
    src = d / "driver.cpp"
    src.write_text(DRIVER)
    exe = d / "driver"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, str(src),
                    os.path.join(CSRC, "tie_order.cpp"), "-o", str(exe), "-lpthread"], check=True)
    return d, exe


def _run(driver, v, t, scale=1.0, threads=0):
    d, exe = driver
    inp, out = d / "mesh.bin", d / "rank.bin"
    with open(inp, "wb") as f:
        np.array([len(v), len(t)], np.int64).tofile(f)
        np.ascontiguousarray(v, np.float32).tofile(f)
        np.ascontiguousarray(t, np.uint32).tofile(f)
    subprocess.run([str(exe), str(inp), str(out), repr(float(scale)), str(threads)], check=True)
    raw = np.fromfile(out, dtype="<i4")
    return bool(raw[0]), raw[1:]


def _walk(links):
    """Slots in the reference walk's order: pop, leaf -> its slots, inner -> push
    left then right."""
    seq, st = [], [0]
    while st:
        left, right, first, count = links[st.pop()]
        if count > 0:
            seq.extend(range(first, first + count))
        else:
            st.append(left)
            st.append(right)
    return np.array(seq)


def _twin_mesh(seed=3):
    """Icosphere with every third triangle also present reversed, in shuffled order."""
    v, t = M.icosphere(3, 1.0)
    rev = t[::3][:, [0, 2, 1]]
    allt = np.concatenate([t, rev])
    return v, allt[np.random.default_rng(seed).permutation(len(allt))]


@pytest.mark.parametrize("kind", ["twins", "icosphere", "trihedral", "plates"])
def test_rank_order_is_the_reference_walk_order(driver, oracle, kind):
    if kind == "twins":
        v, t = _twin_mesh()
    elif kind == "icosphere":
        v, t = M.icosphere(4, 1.0)
    elif kind == "trihedral":
        v, t = M.trihedral(1.0, 10)
    else:
        v, t = M.plate_cluster(40, 4)
    scale = 0.37 if kind == "icosphere" else 1.0
    _, links, order = oracle.build_tree(v, t, scale)
    want = order[_walk(links)]  # caller triangle per walk position
    for threads in (1, 0):
        _, rank = _run(driver, v, t, scale, threads)
        assert np.array_equal(np.argsort(rank), want), (kind, threads)


def test_rank_order_equals_the_reference_builder_on_its_models(driver, oracle):
    import sagittasbr_b200 as sbr
    root = oracle.ref_tree_root()
    if root is None or not oracle.ref_available(64):
        pytest.skip("the reference's builder is built only where the reference tree is present")
    d = os.path.join(root, "assets", "test_models")
    models = sorted(m for m in os.listdir(d) if m.endswith(".obj"))
    assert len(models) >= 6
    found = []
    for m in models:
        v, t = sbr.load_model(os.path.join(d, m))
        v, t = np.asarray(v, np.float32), np.asarray(t, np.int64)
        _, links, tv = oracle.build_tree(v, t, 1.0, source="ref")
        want = tv[_walk(links)]  # the reference's triangles (FP64 vertices) in walk order
        twins, rank = _run(driver, v, t)
        got = (v.astype(np.float64)[t]).reshape(len(t), 9)[np.argsort(rank)]
        assert np.array_equal(got, want), m
        if twins:
            found.append(m)
    assert found == ["b1b.obj", "x35.obj"]


def test_twin_detection(driver):
    v, t = M.icosphere(2, 1.0)
    assert not _run(driver, v, t)[0]
    assert not _run(driver, v, np.concatenate([t, t[:5]]))[0]                    # same winding
    assert not _run(driver, v, np.concatenate([t, t[:5][:, [1, 2, 0]]]))[0]       # rotated: same winding
    assert _run(driver, v, np.concatenate([t, t[7:8][:, [0, 2, 1]]]))[0]          # reversed
    assert _run(driver, v, np.concatenate([t, t[7:8][:, [2, 1, 0]]]))[0]          # reversed
    deg = np.array([[0, 0, 1], [0, 1, 0]], np.uint32)                               # repeated vertex
    assert not _run(driver, v, np.concatenate([t, deg]))[0]
