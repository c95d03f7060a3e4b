"""CPU tests of the glTF 2.0 reader (sbr_load_gltf / sbr_load_model), which follows
the reference's tinygltf-based loader (src/modelLoader.cpp:286-413): TRIANGLES
primitives of every mesh in file order, FLOAT positions, u8 / u16 / u32 or absent
indices, per-primitive vertex offsets, strides and offsets honoured, node
transforms ignored.  Fixtures are written by the test itself."""
import base64
import json
import struct

import numpy as np
import pytest

import sagittasbr_b200 as sbr


def _scene(tmp_path, kind="external"):
    """Two meshes: a quad (u16 indices, interleaved position+normal with stride 24),
    a triangle fan without indices; plus a LINES primitive and an int16 POSITION
    primitive that must be skipped, and a u8-indexed triangle."""
    quad = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    normals = np.tile(np.array([0, 0, 1], np.float32), (4, 1))
    inter = np.concatenate([quad, normals], axis=1).astype(np.float32)        # stride 24
    qidx = np.array([0, 1, 2, 0, 2, 3], np.uint16)
    tri2 = np.array([[0, 0, 1], [1, 0, 1], [0, 1, 1], [1, 1, 1], [2, 0, 1], [2, 1, 1]], np.float32)
    tri3 = np.array([[5, 5, 5], [6, 5, 5], [5, 6, 5]], np.float32)
    i3 = np.array([0, 1, 2], np.uint8)
    lines = np.array([[9, 9, 9], [8, 8, 8]], np.float32)
    ipos = np.array([[1, 2, 3], [4, 5, 6], [7, 8, 9]], np.int16)
    chunks = [(b"\x00" * 4), inter.tobytes(), qidx.tobytes(), b"\x00\x00", tri2.tobytes(), tri3.tobytes(),
              i3.tobytes(), b"\x00", lines.tobytes(), ipos.tobytes(), b"\x00\x00"]
    blob = b"".join(chunks)
    o = np.cumsum([0] + [len(c) for c in chunks])
    views = [
        {"buffer": 0, "byteOffset": int(o[1]), "byteLength": inter.nbytes, "byteStride": 24},
        {"buffer": 0, "byteOffset": int(o[2]), "byteLength": qidx.nbytes},
        {"buffer": 0, "byteOffset": int(o[4]), "byteLength": tri2.nbytes},
        {"buffer": 0, "byteOffset": int(o[5]), "byteLength": tri3.nbytes},
        {"buffer": 0, "byteOffset": int(o[6]), "byteLength": i3.nbytes},
        {"buffer": 0, "byteOffset": int(o[8]), "byteLength": lines.nbytes},
        {"buffer": 0, "byteOffset": int(o[9]), "byteLength": ipos.nbytes},
    ]
    accs = [
        {"bufferView": 0, "componentType": 5126, "count": 4, "type": "VEC3"},                    # 0 quad pos
        {"bufferView": 0, "byteOffset": 12, "componentType": 5126, "count": 4, "type": "VEC3"},  # 1 normals
        {"bufferView": 1, "componentType": 5123, "count": 6, "type": "SCALAR"},                  # 2 u16
        {"bufferView": 2, "componentType": 5126, "count": 6, "type": "VEC3"},                    # 3 no index
        {"bufferView": 3, "componentType": 5126, "count": 3, "type": "VEC3"},                    # 4
        {"bufferView": 4, "componentType": 5121, "count": 3, "type": "SCALAR"},                  # 5 u8
        {"bufferView": 5, "componentType": 5126, "count": 2, "type": "VEC3"},                    # 6 lines
        {"bufferView": 6, "componentType": 5122, "count": 3, "type": "VEC3"},                    # 7 int16
    ]
    doc = {
        "asset": {"version": "2.0"},
        "nodes": [{"mesh": 0, "translation": [100, 0, 0]}],
        "meshes": [
            {"primitives": [{"attributes": {"POSITION": 0, "NORMAL": 1}, "indices": 2},
                            {"attributes": {"POSITION": 6}, "mode": 1},
                            {"attributes": {"POSITION": 3}}]},
            {"primitives": [{"attributes": {"POSITION": 7}},
                            {"attributes": {"POSITION": 4}, "indices": 5, "mode": 4}]},
        ],
        "accessors": accs, "bufferViews": views,
        "buffers": [{"byteLength": len(blob)}],
    }
    want_v = np.concatenate([quad, tri2, tri3])
    want_t = np.array([[0, 1, 2], [0, 2, 3], [4, 5, 6], [7, 8, 9], [10, 11, 12]], np.uint32)
    if kind == "external":
        (tmp_path / "m.bin").write_bytes(blob)
        doc["buffers"][0]["uri"] = "m.bin"
        path = tmp_path / "m.gltf"
        path.write_text(json.dumps(doc))
    elif kind == "datauri":
        doc["buffers"][0]["uri"] = "data:application/octet-stream;base64," + base64.b64encode(blob).decode()
        path = tmp_path / "m.gltf"
        path.write_text(json.dumps(doc, indent=2))
    else:
        js = json.dumps(doc).encode()
        js += b" " * (-len(js) % 4)
        bn = blob + b"\x00" * (-len(blob) % 4)
        body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(bn), 0x004E4942) + bn
        path = tmp_path / "m.glb"
        path.write_bytes(struct.pack("<4sII", b"glTF", 2, 12 + len(body)) + body)
    return str(path), want_v, want_t


@pytest.mark.parametrize("kind", ["external", "datauri", "glb"])
def test_gltf_reader_matches_reference_rules(tmp_path, kind):
    path, want_v, want_t = _scene(tmp_path, kind)
    v, t = sbr.load_gltf(path)
    np.testing.assert_array_equal(v, want_v)
    np.testing.assert_array_equal(t, want_t)
    v2, t2 = sbr.load_model(path)
    np.testing.assert_array_equal(v2, v)
    np.testing.assert_array_equal(t2, t)


def test_gltf_errors(tmp_path):
    with pytest.raises(sbr.SbrError) as e:
        sbr.load_gltf(str(tmp_path / "missing.gltf"))
    assert e.value.status == 12
    bad = tmp_path / "bad.gltf"
    bad.write_text('{"asset": {"version": "2.0"}, "meshes": [')
    with pytest.raises(sbr.SbrError) as e:
        sbr.load_gltf(str(bad))
    assert e.value.status == 13
    empty = tmp_path / "empty.gltf"
    empty.write_text('{"asset": {"version": "2.0"}}')
    with pytest.raises(sbr.SbrError) as e:
        sbr.load_gltf(str(empty))
    assert e.value.status == 2
    # accessor reaching past its buffer view
    path, _, _ = _scene(tmp_path, "external")
    doc = json.loads(open(path).read())
    doc["accessors"][0]["count"] = 400
    over = tmp_path / "over.gltf"
    over.write_text(json.dumps(doc))
    with pytest.raises(sbr.SbrError) as e:
        sbr.load_gltf(str(over))
    assert e.value.status == 13
    with pytest.raises(sbr.SbrError) as e:
        sbr.load_model(str(tmp_path / "model.stl"))
    assert e.value.status == 14


def test_obj_and_gltf_give_the_same_mesh(tmp_path):
    from sagittasbr_b200 import meshes as M
    v, t = M.icosphere(2)
    obj = tmp_path / "s.obj"
    obj.write_text("".join(f"v {a:.9g} {b:.9g} {c:.9g}\n" for a, b, c in v) +
                   "".join(f"f {a + 1} {b + 1} {c + 1}\n" for a, b, c in t))
    blob = v.astype(np.float32).tobytes() + t.astype(np.uint32).tobytes()
    doc = {"asset": {"version": "2.0"},
           "meshes": [{"primitives": [{"attributes": {"POSITION": 0}, "indices": 1}]}],
           "accessors": [{"bufferView": 0, "componentType": 5126, "count": len(v), "type": "VEC3"},
                         {"bufferView": 1, "componentType": 5125, "count": t.size, "type": "SCALAR"}],
           "bufferViews": [{"buffer": 0, "byteOffset": 0, "byteLength": v.size * 4},
                           {"buffer": 0, "byteOffset": v.size * 4, "byteLength": t.size * 4}],
           "buffers": [{"byteLength": len(blob),
                        "uri": "data:application/octet-stream;base64," + base64.b64encode(blob).decode()}]}
    g = tmp_path / "s.gltf"
    g.write_text(json.dumps(doc))
    vo, to = sbr.load_model(str(obj))
    vg, tg = sbr.load_model(str(g))
    np.testing.assert_array_equal(vo, vg)
    np.testing.assert_array_equal(to, tg)
