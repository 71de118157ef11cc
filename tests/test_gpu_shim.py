"""The drop-in boundary on the GPU: Radia's own module, compiled from the
reference core with this library as its GPU plugin, against its own CPU path.

Each case runs in a child process (tests/shim_cases.py), as a user's fresh
``import radia`` would.  Tolerances: the field of a given magnetization 1e-9
relative (the reference's GPU-vs-CPU FP64 bar, its tests/test_gpu_fld_fp32.py:71),
FP32 field terms 5e-4 (:72); relaxed models 5e-6 relative in B for linear and
5e-5 for saturating materials (its tests/test_recmag_asm.py:134-157), both as
the max-norm ratio and per point (|dB_i| / |B_i|, points with |B_i| below
1e-3 of the largest measured against that floor).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from radiacuda_b200 import refmodule

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["magnet_array", "mixed_sym_m9", "mixed_sym_m11", "iron_dipole_m11", "symmetry_mix",
         "single_precision_field", "srcobj", "cpu_assembly_gpu_relax", "material_change", "direct_solve",
         "table_m9", "table_m11"]


@pytest.fixture(scope="module")
def shim(cuda):
    if not os.path.exists(refmodule.module_path()):
        pytest.fail("radia module with the b200 plugin is not built (radiacuda_b200/shim/Makefile)")
    r = subprocess.run([sys.executable, os.path.join(HERE, "shim_cases.py")] + CASES, capture_output=True,
                       text=True, timeout=1200)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("SHIM_JSON ")]
    assert r.returncode == 0 and line, r.stdout[-3000:] + r.stderr[-3000:]
    # the plugin reports on stderr whenever it declines or fails
    assert "radiacuda_b200" not in r.stderr, r.stderr[-3000:]
    return json.loads(line[0][len("SHIM_JSON "):])


def _errs(got, exp):
    g = np.asarray(got, dtype=float).reshape(-1, 3)
    e = np.asarray(exp, dtype=float).reshape(-1, 3)
    d = np.linalg.norm(g - e, axis=1)
    n = np.linalg.norm(e, axis=1)
    floor = 1e-3 * n.max()
    return float(np.abs(g - e).max() / np.abs(e).max()), float((d / np.maximum(n, floor)).max())


def _check_pair(c, tol):
    assert c["asm_gpu"] == "gpu" and c["fld_gpu"] == "gpu" and c["asm_cpu"] == "cpu" and c["fld_cpu"] == "cpu"
    field_err = _errs(c["b_gpu"], c["b_gpuM_cpu"])
    assert field_err[0] < 1e-9 and field_err[1] < 1e-9, field_err
    solve_err = _errs(c["b_gpu"], c["b_cpu"])
    assert solve_err[0] < tol and solve_err[1] < tol, solve_err
    assert c["st_gpu"][0] <= 1e-9 or c["st_gpu"][0] < c["st_cpu"][0] * 10, (c["st_gpu"], c["st_cpu"])


def test_magnet_array_anisotropic_relaxes_on_the_gpu(shim):
    _check_pair(shim["magnet_array"], 5e-6)


@pytest.mark.parametrize("case", ["mixed_sym_m9", "mixed_sym_m11", "iron_dipole_m11", "table_m9", "table_m11"])
def test_saturating_models_methods_9_and_11(shim, case):
    _check_pair(shim[case], 5e-5)


def test_mixed_symmetry_planes_and_default_randomization(shim):
    c = shim["symmetry_mix"]
    _check_pair(c, 5e-5)
    assert _errs(c["b_gpu"], c["b_cpu"])[0] < 1e-6


def test_single_precision_field_option(shim):
    c = shim["single_precision_field"]
    assert c["fld_f32"] == "gpu"
    assert _errs(c["b_f32"], c["b_cpu"])[0] < 5e-4


def test_frozen_source_object(shim):
    c = shim["srcobj"]
    assert c["asm_gpu"] == "gpu"
    assert _errs(c["b_gpu"], c["b_cpu"])[0] < 5e-5


def test_cpu_assembled_matrix_relaxed_on_the_gpu(shim):
    c = shim["cpu_assembly_gpu_relax"]
    assert c["asm"] == "cpu"
    assert _errs(c["b_gpu"], c["b_cpu"])[0] < 5e-6


def test_material_change_after_rlxpre(shim):
    c = shim["material_change"]
    assert _errs(c["b_gpu"], c["b_cpu"])[0] < 5e-6


def test_device_direct_solve_through_the_module(shim):
    c = shim["direct_solve"]
    assert c["asm_gpu"] == "gpu"
    assert c["st_f64"][0] < 1e-12 and c["st_tf32"][0] < 1e-12, (c["st_f64"], c["st_tf32"])
    for k in ("b_f64", "b_tf32"):
        assert _errs(c[k], c["b_cpu"])[0] < 5e-6, k
