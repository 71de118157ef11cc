"""The drop-in boundary without a GPU: Radia's own module built with this
library as its GPU plugin loads, defines every radGPU_* symbol its core calls
(cpp/src/core/radgpu_asm.h:149-187, radrlmet.h:700-702, radgpu_fld.h:184,198
of the reference), and, where no device exists, declines every GPU request
so that the core's CPU path gives the same results (or raises under
UtiGpuFallback('break')) -- the reference's own contract for a failing GPU."""
import json
import os
import re
import subprocess
import sys

import pytest

from radiacuda_b200 import refmodule

HERE = os.path.dirname(os.path.abspath(__file__))

SEAM = ["radGPU_PackGeometryForAsm", "radGPU_PackObsQuadForAsm", "radGPU_AssembleMatrix", "radGPU_FreeAsmData",
        "radGPU_FreeSymData", "radGPU_FreeObsQuadData", "radGPU_PublishAssembledMatrix",
        "radGPU_DiscardAssembledMatrix", "radGPU_AutoRelax", "radGPU_AutoRelaxNK", "radGPU_PackInteractionData",
        "radGPU_UnpackMagnetization", "radGPU_ComputeField", "radGPU_ComputeFieldFromSrcRep"]


def _module():
    p = refmodule.module_path()
    if not os.path.exists(p):
        pytest.skip("radia module with the b200 plugin not built (needs the reference sources)")
    return p


def test_module_defines_the_seam():
    p = _module()
    out = subprocess.run(["nm", "-DC", "--defined-only", p], capture_output=True, text=True).stdout
    defined = set(re.findall(r" T (radGPU_\w+)\(", out))
    assert set(SEAM) <= defined, set(SEAM) - defined
    assert " T radB200_DirectSolve" in out
    # the plugin links this library, not the reference's CUDA objects
    deps = subprocess.run(["ldd", p], capture_output=True, text=True).stdout
    assert "libradb200.so" in deps


def test_without_a_device_the_core_falls_back_and_break_raises():
    _module()
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU path runs (tests/test_gpu_shim.py)")
    r = subprocess.run([sys.executable, os.path.join(HERE, "shim_cases.py"), "break_policy"], capture_output=True,
                       text=True, timeout=600)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("SHIM_JSON ")]
    assert r.returncode == 0 and line, r.stdout + r.stderr
    c = json.loads(line[0][len("SHIM_JSON "):])["break_policy"]
    assert "Error602" in c["raised"] or "GPU" in c["raised"], c
    assert c["asm"] == "cpu" and c["policy"] == "cpu"
    assert c["st"][0] < 1e-10
    assert "radiacuda_b200 assembly failed" in r.stderr
