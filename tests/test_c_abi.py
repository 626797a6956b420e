"""A non-Python caller on the boundary: tests/c/xk_abi_check.c is compiled
with gcc against include/xk.h and linked to libxk.so, then run on the
reference's fixture (validation/fixtures/diffraction_ref.json).

Without a GPU it must report XK_ERR_NO_DEVICE from xk_init and
xk_kirchhoff_auto (there is no CPU fallback). On the GPU its
xk_diffraction_integral results must match the fixture (abs 1e-10 on
XK_PATH_F64, rel L2 1e-4 on XK_PATH_F32PR) and its xk_kirchhoff_gpu
results the oracle's plain FP64 sum of the f32 records (1e-4 per pixel,
tests/golden_gpu_kirchhoff.rs:103-182)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "xk_abi_check.c")
LIBDIR = os.path.join(ROOT, "xrt-rs_b200")


def _build(tmp_path):
    gcc = shutil.which("gcc") or shutil.which("cc")
    if gcc is None:
        pytest.skip("no C compiler")
    if not os.path.exists(os.path.join(LIBDIR, "libxk.so")):
        pytest.fail("libxk.so is not built")
    exe = str(tmp_path / "xk_abi_check")
    subprocess.run([gcc, "-std=c11", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "include"), SRC, "-L", LIBDIR, "-lxk",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def _case_file(tmp_path, golden_case):
    r = golden_case["rays"]
    p = golden_case["pixels"]
    lines = [str(len(r["x"]))]
    lines += [" ".join(repr(float(v)) for v in r[k]) for k in cases.RAY_FIELDS]
    lines.append(str(len(p["x"])))
    lines += [" ".join(repr(float(v)) for v in p[k]) for k in cases.PIXEL_FIELDS]
    path = tmp_path / "case.txt"
    path.write_text("\n".join(lines) + "\n")
    return str(path)


def _run(exe, case):
    r = subprocess.run([exe, case], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = {}
    for line in r.stdout.splitlines():
        parts = line.split()
        if parts[0] in ("f64", "f32pr", "gpu"):
            rows.setdefault(parts[0], []).append([float(v) for v in parts[2:6]])
    return r.stdout, {k: np.array(v) for k, v in rows.items()}


def test_c_caller_builds_and_reports_no_device_or_runs(tmp_path, golden_case):
    exe = _build(tmp_path)
    out, rows = _run(exe, _case_file(tmp_path, golden_case))
    assert out.startswith("version ")
    assert "no-device" in out or "done" in out


@pytest.mark.gpu
def test_c_caller_matches_fixture_and_oracle(tmp_path, golden_case, oracle):
    exe = _build(tmp_path)
    out, rows = _run(exe, _case_file(tmp_path, golden_case))
    assert "done" in out, out
    exp = np.array([[e[c] for c in ("es_re", "es_im", "ep_re", "ep_im")]
                    for e in golden_case["expected"]])
    assert np.max(np.abs(rows["f64"] - exp)) < 1e-10
    got = rows["f32pr"][:, 0] + 1j * rows["f32pr"][:, 1]
    ref = exp[:, 0] + 1j * exp[:, 1]
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-4
    r = golden_case["rays"]
    f32 = [np.asarray(r[k], dtype=np.float32).astype(np.float64) for k in cases.RAY_FIELDS]
    pix = [np.asarray(golden_case["pixels"][k], dtype=np.float32).astype(np.float64)
           for k in "xyz"]
    plain = oracle.plain_f64(f32, pix)
    for i in range(len(pix[0])):
        c = plain[0][i] + 1j * plain[1][i]
        g = rows["gpu"][i, 0] + 1j * rows["gpu"][i, 1]
        assert abs(g - c) / abs(c) < 1e-4
