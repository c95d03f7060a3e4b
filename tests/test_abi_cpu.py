"""CPU tests of the C ABI boundary: the library loads, exports every function
include/sbr.h declares, its struct layouts agree with the ctypes mirror, and the
host-side entry surface (config.txt, OBJ, CSV) behaves like the reference's.
No GPU compute is called here."""
import ctypes as C
import json
import os
import re
import subprocess

import numpy as np
import pytest

import sagittasbr_b200 as sbr
from sagittasbr_b200 import _lib

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HEADER = os.path.join(ROOT, "include", "sbr.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sbr_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    L = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the ctypes mirror declares exactly these
    assert set(names) == set(_lib.SIGNATURES)


def test_struct_layouts_match_header(tmp_path):
    structs = {
        "sbr_build_opts": _lib.BuildOpts, "sbr_scene_info": _lib.SceneInfo, "sbr_job": _lib.Job,
        "sbr_run_opts": _lib.RunOpts, "sbr_result": _lib.Result, "sbr_plan_info": _lib.PlanInfo,
        "sbr_config": _lib.Config,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sbr.h"', "int main(void){", 'printf("{");']
    first = True
    for cname, py in structs.items():
        for f, _ in py._fields_:
            sep = "" if first else ","
            first = False
            lines.append(f'printf("{sep}\\"{cname}.{f}\\": %zu", offsetof({cname}, {f}));')
        lines.append(f'printf(",\\"{cname}\\": %zu", sizeof({cname}));')
    lines.append(f'printf(",\\"sbr_ray_record\\": %zu", sizeof(sbr_ray_record));')
    lines.append('printf("}\\n"); return 0; }')
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = json.loads(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    for cname, py in structs.items():
        assert got[cname] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[f"{cname}.{f}"] == getattr(py, f).offset, f"{cname}.{f}"
    assert got["sbr_ray_record"] == sbr.RAY_RECORD.itemsize


def test_constants_match_header(tmp_path):
    """The ctypes mirror's mode, precision, polarisation and first-hit constants are
    the header's."""
    names = ["SBR_MODE_BATCHED", "SBR_MODE_PER_ANGLE", "SBR_PREC_MIXED", "SBR_PREC_FP32", "SBR_PREC_FP64",
             "SBR_POL_SCALAR", "SBR_POL_HHVV", "SBR_FIRST_HIT_AUTO", "SBR_FIRST_HIT_RASTER",
             "SBR_FIRST_HIT_TRAVERSE"]
    lines = ['#include <stdio.h>', '#include "sbr.h"', "int main(void){"]
    lines += [f'printf("%d\\n", (int){n});' for n in names]
    lines.append("return 0; }")
    src = tmp_path / "consts.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "consts"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [getattr(_lib, n[4:]) for n in names]
    assert got == want


def test_status_strings():
    L = _lib.lib()
    assert L.sbr_status_str(0) == b"SBR_OK"
    for code, name in _lib.STATUS_NAMES.items():
        assert L.sbr_status_str(code).decode() == name
    assert L.sbr_status_str(999) == b"SBR_ERR_UNKNOWN"
    assert L.sbr_abi_version() == 3


REF_STYLE_CONFIG = """# angular sampling
phi_start      0        # deg
phi_end        360
phi_samples    30
theta_start    0
theta_end      180
theta_samples  20
freq           1e10     # Hz
grid_size      100
n_x            20000
n_y            20000
tpb_x          16
tpb_y          16
max_bounces    100
reflection_const 1.0
show_info_GPU  1
show_hit_stats 0
"""


def test_config_defaults_when_file_missing(tmp_path, capfd):
    cfg = sbr.load_config(str(tmp_path / "nope.txt"), [])
    assert "Could not open" in capfd.readouterr().err
    assert (cfg["phi_start"], cfg["phi_end"], cfg["phi_samples"]) == (0.0, 180.0, 181)
    assert (cfg["theta_start"], cfg["theta_end"], cfg["theta_samples"]) == (90.0, 90.0, 1)
    assert (cfg["grid_size"], cfg["nx"], cfg["ny"], cfg["max_bounces"]) == (10.0, 5000, 5000, 20)
    assert (cfg["reflection_const"], cfg["freq"], cfg["show_info_gpu"], cfg["show_hit_stats"]) == (1.0, 1e10, 1, 1)
    assert cfg["freq_source"] == 0 and cfg["model_path"] == "" and cfg["model_scale"] == 1.0


def test_config_file_and_cli_precedence(tmp_path, capfd):
    p = tmp_path / "c.txt"
    p.write_text(REF_STYLE_CONFIG)
    cfg = sbr.load_config("config.txt", ["--config", str(p), "--model", "m.obj", "--model-scale", "0.5"])
    assert cfg["phi_end"] == 360.0 and cfg["theta_samples"] == 20 and cfg["nx"] == 20000
    assert cfg["freq"] == 1e10 and cfg["freq_source"] == 1 and cfg["show_hit_stats"] == 0
    assert cfg["model_path"] == "m.obj" and cfg["model_scale"] == 0.5
    # first bare argument is the frequency and wins over the file; unknown flags warn
    cfg = sbr.load_config(str(p), ["2.5e9", "3e9", "--bogus", "--model", "x.obj"])
    assert cfg["freq"] == 2.5e9 and cfg["freq_source"] == 2
    assert "Unrecognized argument '--bogus'" in capfd.readouterr().err
    with pytest.raises(sbr.SbrError):
        sbr.load_config(str(p), ["--model"])


def test_config_angle_grid_is_theta_major(tmp_path):
    p = tmp_path / "c.txt"
    p.write_text("theta_start 10\ntheta_end 30\ntheta_samples 3\nphi_start 0\nphi_end 90\nphi_samples 4\n")
    cfg = sbr.load_config(str(p), [])
    th, ph = sbr.config_angles(cfg)
    np.testing.assert_array_equal(th, np.repeat([10.0, 20.0, 30.0], 4))
    np.testing.assert_array_equal(ph, np.tile([0.0, 30.0, 60.0, 90.0], 3))
    p.write_text("theta_samples 1\ntheta_start 45\nphi_samples 1\nphi_start 7\n")
    th, ph = sbr.config_angles(sbr.load_config(str(p), []))
    assert list(th) == [45.0] and list(ph) == [7.0]


def test_obj_loader_triangulation(tmp_path):
    p = tmp_path / "m.obj"
    p.write_text(
        "# comment\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0 0 1\nvn 0 0 1\nvt 0 0\n"
        "f 1 2 3\n"            # triangle
        "f 1/1/1 2/1/1 3/1/1 4/1/1\n"  # quad: |v3-v1|^2 == |v4-v2|^2 -> split (1,2,4),(2,3,4)
        "f -5 -4 -1\n"         # negative indices: 1 2 5
        "f 1 2 3 4 5\n")       # pentagon: fan
    v, t = sbr.load_obj(str(p))
    assert v.shape == (5, 3)
    assert t.tolist() == [[0, 1, 2], [0, 1, 3], [1, 2, 3], [0, 1, 4], [0, 1, 2], [0, 2, 3], [0, 3, 4]]
    p.write_text("v 0 0 0\nv 1 0 0\nv 2 0 0\nv 0 0 1\nf 1 2 3 4\n")  # shorter diagonal is 1-3? |v3-v1|=2, |v4-v2|=sqrt2
    v, t = sbr.load_obj(str(p))
    assert t.tolist() == [[0, 1, 3], [1, 2, 3]]
    p.write_text("v 0 0 0\nf 1 2 3\n")
    with pytest.raises(sbr.SbrError):
        sbr.load_obj(str(p))
    with pytest.raises(sbr.SbrError):
        sbr.load_obj(str(tmp_path / "missing.obj"))


def test_csv_layout(tmp_path):
    cfg = sbr.load_config(str(tmp_path / "none"), [])
    cfg.update(freq=1e10, nx=10000, ny=10000, grid_size=2.5, theta_samples=1, phi_samples=2)
    out = tmp_path / "rcs_results.csv"
    sbr.write_csv(str(out), cfg, [90.0, 90.0], [0.0, 6.2068965517], [3.152731, 3.1511], [4.986871, 4.984634])
    assert out.read_text().splitlines() == [
        "# Frequency: 1e+10", "# Grid: 10000x10000", "# GridSize: 2.5", "# ThetaSamples: 1", "# PhiSamples: 2",
        "theta,phi,rcs_m2,rcs_dbsm", "90,0,3.15273,4.98687", "90,6.2069,3.1511,4.98463"]


def test_csv_full_precision_round_trips(tmp_path):
    """csv_digits 17 (config key or --full-precision) writes rows that read back to the
    same doubles; the header keeps the reference's formatting."""
    (tmp_path / "config.txt").write_text("csv_digits 17\n")
    cfg = sbr.load_config(str(tmp_path / "config.txt"), [])
    assert cfg["csv_digits"] == 17
    assert sbr.load_config(str(tmp_path / "none"), ["--full-precision"])["csv_digits"] == 17
    cfg.update(freq=1e10, nx=10000, ny=10000, grid_size=2.5, theta_samples=1, phi_samples=2)
    vals = np.array([[90.0, 0.1 + 0.2, np.pi, 10 * np.log10(np.pi)], [90.0, 6.2068965517241379, 1e-10 / 3, -100.0]])
    out = tmp_path / "rcs_results.csv"
    sbr.write_csv(str(out), cfg, vals[:, 0], vals[:, 1], vals[:, 2], vals[:, 3])
    lines = out.read_text().splitlines()
    assert lines[0] == "# Frequency: 1e+10"
    back = np.array([[float(x) for x in ln.split(",")] for ln in lines[6:]])
    assert np.array_equal(back, vals)
    cfg["csv_digits"] = 18
    with pytest.raises(sbr.SbrError):
        sbr.write_csv(str(out), cfg, vals[:, 0], vals[:, 1], vals[:, 2], vals[:, 3])


def test_scene_requires_gpu_or_reports_cleanly():
    """Without a device the library reports SBR_ERR_NO_DEVICE (never a CPU fallback);
    invalid meshes are rejected before any device work."""
    from sagittasbr_b200 import meshes as M
    v, t = M.box()
    with pytest.raises(sbr.SbrError) as e:
        sbr.Scene(v, np.zeros((0, 3), np.uint32))
    assert e.value.status == 2  # SBR_ERR_EMPTY_MESH
    with pytest.raises(sbr.SbrError) as e:
        sbr.Scene(v, np.array([[0, 1, 99]], np.uint32))
    assert e.value.status == 3  # SBR_ERR_BAD_INDEX
    bad = v.copy()
    bad[0, 0] = np.nan
    with pytest.raises(sbr.SbrError) as e:
        sbr.Scene(bad, t)
    assert e.value.status == 4  # SBR_ERR_NONFINITE
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(sbr.SbrError) as e:
            sbr.Scene(v, t)
        assert e.value.status == 8  # SBR_ERR_NO_DEVICE


def test_reference_gpu_build_loads():
    """The reference's own GPU sweep (built into baseline/_ref by baseline/Makefile
    where the reference tree is present) loads and reports its precision."""
    from baseline import ref_gpu
    for bits in (32, 64):
        if not ref_gpu.available(bits):
            pytest.skip("reference GPU build not present")
        assert ref_gpu.lib(bits).sbrref_gpu_real_bits() == bits


def test_csv_error_column(tmp_path):
    """error_bound 1 (config key): rcs_results.csv gains a fifth column rcs_err_db;
    without it the layout is the reference's."""
    (tmp_path / "config.txt").write_text("error_bound 1\nphi_samples 2\n")
    cfg = sbr.load_config(str(tmp_path / "config.txt"))
    assert cfg["error_bound"] == 1
    assert sbr.load_config(str(tmp_path / "none"))["error_bound"] == 0
    th, ph = np.array([90.0, 90.0]), np.array([0.0, 180.0])
    p = tmp_path / "rcs_results.csv"
    sbr.write_csv(str(p), cfg, th, ph, np.array([1.0, 2.0]), np.array([0.0, 3.0103]), np.array([0.01, 0.25]))
    lines = p.read_text().splitlines()
    assert lines[5] == "theta,phi,rcs_m2,rcs_dbsm,rcs_err_db"
    assert lines[6].split(",")[-1] == "0.01" and lines[7].split(",")[-1] == "0.25"
    sbr.write_csv(str(p), cfg, th, ph, np.array([1.0, 2.0]), np.array([0.0, 3.0103]))
    assert p.read_text().splitlines()[5] == "theta,phi,rcs_m2,rcs_dbsm"
