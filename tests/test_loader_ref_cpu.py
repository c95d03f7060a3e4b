"""The model loaders pinned to the reference's OWN loader (CPU).

oracle/_ref/libsbrrefload.so is src/modelLoader.cpp (with its vendored
tinyobjloader / tinygltf) compiled for the host from where it lies, behind a shim
that de-indexes the mesh with the model scale as runRcsApp does in its FP32 build
(src/app/rtRcsEntry.cu:108-145).  sbr_load_model's triangles, de-indexed the same
way (float32 position x float32 scale), must equal them byte for byte:

* on every OBJ model the reference ships (assets/test_models: quads split along the
  shorter diagonal in FP32, as tinyobjloader does; de-duplicated vertices), also
  against the committed digests in tests/golden/loader_ref.json
  (tests/golden/make_loader_golden.py);
* on the glTF / GLB scenes of test_gltf_cpu.py (external buffer, data URI, binary).

The reference tree is read where oracle/_ref was built from it (oracle/_ref/ref_root.txt).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import sagittasbr_b200 as sbr

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def ref(oracle):
    if not os.path.exists(oracle.REF_LOAD_SO) or oracle.ref_tree_root() is None:
        pytest.skip("the reference loader is built only where the reference tree is present")
    return oracle


def _ours(path, scale):
    v, t = sbr.load_model(path)
    return (np.asarray(v, np.float32) * np.float32(scale))[np.asarray(t, np.int64)]


def _models(ref):
    d = os.path.join(ref.ref_tree_root(), "assets", "test_models")
    return [os.path.join(d, m) for m in sorted(os.listdir(d)) if m.endswith(".obj")]


@pytest.mark.parametrize("scale", [1.0, 0.37])
def test_obj_models_equal_reference_loader(ref, scale):
    golden = json.load(open(os.path.join(HERE, "golden", "loader_ref.json")))
    models = _models(ref)
    assert len(models) >= 6
    for path in models:
        want = ref.ref_load_triangles(path, scale)
        got = _ours(path, scale)
        assert got.shape == want.shape, path
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), path
        g = golden[os.path.basename(path)][f"{scale:g}"]
        assert g["triangles"] == got.shape[0]
        assert hashlib.sha256(got.astype("<f4").tobytes()).hexdigest() == g["sha256"], path


@pytest.mark.parametrize("kind", ["external", "datauri", "glb"])
def test_gltf_equals_reference_loader(ref, tmp_path, kind):
    from test_gltf_cpu import _scene
    path, _, _ = _scene(tmp_path, kind)
    want = ref.ref_load_triangles(path, 1.0)
    got = _ours(path, 1.0)
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
