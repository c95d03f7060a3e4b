"""GPU checks of the entry surface: the RT-RCS drop-in with OBJ and glTF models, its
frequency-scan mode against the Python driver and the Mie series, and the
per-angle hit statistics it prints."""
import base64
import json
import os
import subprocess

import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import meshes as M

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
CLI = os.path.join(ROOT, "sagittasbr_b200", "bin", "RT-RCS")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def _write_obj(path, v, t):
    with open(path, "w") as f:
        f.writelines(f"v {a:.9g} {b:.9g} {c:.9g}\n" for a, b, c in v)
        f.writelines(f"f {a + 1} {b + 1} {c + 1}\n" for a, b, c in t)


def _write_gltf(path, v, t):
    blob = v.astype(np.float32).tobytes() + t.astype(np.uint32).tobytes()
    doc = {"asset": {"version": "2.0"},
           "meshes": [{"primitives": [{"attributes": {"POSITION": 0}, "indices": 1}]}],
           "accessors": [{"bufferView": 0, "componentType": 5126, "count": len(v), "type": "VEC3"},
                         {"bufferView": 1, "componentType": 5125, "count": t.size, "type": "SCALAR"}],
           "bufferViews": [{"buffer": 0, "byteOffset": 0, "byteLength": v.size * 4},
                           {"buffer": 0, "byteOffset": v.size * 4, "byteLength": t.size * 4}],
           "buffers": [{"byteLength": len(blob),
                        "uri": "data:application/octet-stream;base64," + base64.b64encode(blob).decode()}]}
    with open(path, "w") as f:
        json.dump(doc, f)


CONFIG = """phi_start 0
phi_end 350
phi_samples 36
theta_start 90
theta_end 90
theta_samples 1
grid_size 2.2
n_x 240
n_y 240
max_bounces 3
reflection_const 1.0
freq 1e9
show_hit_stats 1
"""


def test_cli_obj_and_gltf_and_hit_stats(tmp_path):
    v, t = M.icosphere(4, 1.0)
    _write_obj(tmp_path / "s.obj", v, t)
    _write_gltf(tmp_path / "s.gltf", v, t)
    (tmp_path / "config.txt").write_text(CONFIG)
    out = {}
    for m in ("s.obj", "s.gltf"):
        p = subprocess.run([CLI, "--model", m], cwd=tmp_path, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        out[m] = (tmp_path / "rcs_results.csv").read_text()
        assert p.stderr.count("| Hit:") == 36
    assert out["s.obj"] == out["s.gltf"]
    rows = [r for r in out["s.obj"].splitlines() if r and not r.startswith("#")]
    assert rows[0] == "theta,phi,rcs_m2,rcs_dbsm" and len(rows) == 37


def test_cli_frequency_scan_matches_python_driver_and_mie(tmp_path):
    from oracle import mie
    v, t = M.icosphere(5, 1.0)
    _write_obj(tmp_path / "s.obj", v, t)
    (tmp_path / "config.txt").write_text(CONFIG)
    p = subprocess.run([CLI, "--model", "s.obj", "--freq-scan", "1e9", "3e9", "5"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    lines = (tmp_path / "results_freq_scans.csv").read_text().splitlines()
    assert lines[0] == "Frequency,Avg_RCS,Std_RCS" and len(lines) == 6
    cli = np.array([[float(x) for x in r.split(",")] for r in lines[1:]])
    cfg = sbr.load_config(str(tmp_path / "config.txt"))
    with sbr.Scene(v, t) as sc:
        fr, mean, std = sbr.freq_scan(cfg, sc, 1e9, 3e9, 5, out_csv=None)
        # the same frequencies traced one at a time
        th, ph = sbr.config_angles(cfg)
        one = [sbr.run(sc, sbr.JobSpec(th, ph, [f], 240, 240, 2.2, 3)).sigma_m2.mean() for f in fr]
    np.testing.assert_array_equal(cli[:, 0], fr)
    np.testing.assert_allclose(cli[:, 1], mean, rtol=1e-12)
    np.testing.assert_allclose(cli[:, 2], std, rtol=1e-9)
    # the 5-frequency trace sums each 4x8 ray block in FP32 first (lane-owned
    # epilogue), the 1-frequency traces sum in FP64
    np.testing.assert_allclose(mean, one, rtol=1e-5)
    mie_sigma = np.array([mie.sphere_rcs(1.0, f) for f in fr])
    assert np.all(np.abs(mean / mie_sigma - 1.0) < 0.15), mean / mie_sigma


def test_frequency_scan_with_more_than_128_frequencies():
    v, t = M.icosphere(3, 1.0)
    cfg = {"phi_start": 0.0, "phi_end": 90.0, "phi_samples": 4, "theta_start": 90.0, "theta_end": 90.0,
           "theta_samples": 1, "grid_size": 2.2, "nx": 64, "ny": 64, "max_bounces": 2, "reflection_const": 1.0}
    with sbr.Scene(v, t) as sc:
        fr, mean, std = sbr.freq_scan(cfg, sc, 1e8, 1e9, 130, out_csv=None)
        th, ph = sbr.config_angles(cfg)
        ref = sbr.run(sc, sbr.JobSpec(th, ph, fr[128:], 64, 64, 2.2, 2)).sigma_m2.reshape(4, 2).mean(axis=0)
    assert fr.size == 130 and mean.size == 130
    # the scan's plan holds a 128-frequency job, so its 2-frequency job is summed in
    # the lane-owned layout (FP32 block partials) and its own run per lane in FP64
    np.testing.assert_allclose(mean[128:], ref, rtol=1e-5)
