"""Cases for the drop-in boundary tests, run in a child process.

Radia's own module, built from the reference core with this library as its
GPU plugin (radiacuda_b200.refmodule), solves and evaluates each model twice:
through the GPU path (RlxPre/Fld use_gpu=True, RlxAuto methods 9 and 11,
or the device direct solve) and through the same module's CPU path
(use_gpu=False, method 4).  It prints one JSON object with the backends the
module reported and the fields of both paths.

    python tests/shim_cases.py <case> [<case> ...]
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import models as MD  # noqa: E402
from radiacuda_b200 import refmodule  # noqa: E402

GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))


def _backends(rad):
    return {"asm": rad.UtiAsmLastBackend(), "fld": rad.UtiFldLastBackend()}


def _solve_pair(rad, h, pts, meth_gpu, prec, iters, meth_cpu=4, prec_cpu=None):
    """GPU solve + field, the CPU field of the GPU magnetization, then CPU
    solve + field of the same model."""
    out = {}
    im = rad.RlxPre(h, use_gpu=True)
    out["asm_gpu"] = rad.UtiAsmLastBackend()
    out["st_gpu"] = list(rad.RlxAuto(im, prec, iters, meth_gpu, "ZeroM->True"))
    out["b_gpu"] = rad.Fld(h, "b", pts, use_gpu=True)
    out["fld_gpu"] = rad.UtiFldLastBackend()
    out["b_gpuM_cpu"] = rad.Fld(h, "b", pts, use_gpu=False)
    out["fld_cpu"] = rad.UtiFldLastBackend()
    im2 = rad.RlxPre(h, use_gpu=False)
    out["asm_cpu"] = rad.UtiAsmLastBackend()
    out["st_cpu"] = list(rad.RlxAuto(im2, prec if prec_cpu is None else prec_cpu, 100000, meth_cpu, "ZeroM->True"))
    out["b_cpu"] = rad.Fld(h, "b", pts, use_gpu=False)
    return out


def case_magnet_array(rad):
    """The 432-block anisotropic permanent-magnet array at its 10,000 field
    points (the reference's GPU solver declines anisotropic materials)."""
    h = MD.magnet_array(rad)
    P = MD.magnet_array_points().tolist()
    return _solve_pair(rad, h, P, 9, 1e-11, 2000)


def case_mixed_sym_m9(rad):
    h = MD.mixed_sym(rad)
    return _solve_pair(rad, h, GOLD["cases"]["mixed_sym"]["points"], 9, 1e-10, 5000)


def case_mixed_sym_m11(rad):
    h = MD.mixed_sym(rad)
    return _solve_pair(rad, h, GOLD["cases"]["mixed_sym"]["points"], 11, 1e-10, 5000)


def case_iron_dipole_m11(rad):
    c = GOLD["cases"]["iron_dipole_300"]
    h = MD.iron_dipole(rad, **c["kwargs"])
    h = h[0] if isinstance(h, tuple) else h
    return _solve_pair(rad, h, c["points"], 11, 1e-10, 5000)


def _cluster(rad, rng, n, lo, hi):
    ids = []
    for _ in range(n):
        v = rng.uniform(lo, hi) + rng.uniform(1.5, 7.0, size=(4, 3))
        ids.append(rad.ObjPolyhdr(v.tolist(), MD.TET_FACES))
    return rad.ObjCnt(ids)


def case_symmetry_mix(rad):
    """Tetrahedra under four mirror planes, under one, and under none, with a
    saturating law and a racetrack, at the default length randomization."""
    rad.UtiDelAll()
    rad.FldLenRndSw("on")
    rng = np.random.default_rng(17)
    a = _cluster(rad, rng, 14, [35, 6, 6], [80, 28, 30])
    rad.TrfZerPerp(a, [0, 0, 0], [1, -1, 0])
    rad.TrfZerPerp(a, [0, 0, 0], [1, 0, 0])
    rad.TrfZerPerp(a, [0, 0, 0], [0, 1, 0])
    rad.TrfZerPara(a, [0, 0, 0], [0, 0, 1])
    b = _cluster(rad, rng, 9, [-130, 12, -18], [-95, 38, 18])
    rad.TrfZerPerp(b, [0, 0, 0], [0, 1, 0])
    c = _cluster(rad, rng, 7, [95, 95, -25], [130, 130, 8])
    mat = rad.MatSatIsoFrm([20000, 2], [0.1, 2], [0.1, 2])
    for g in (a, b, c):
        rad.MatApl(g, mat)
    coil = rad.ObjRaceTrk([0, 0, 45], [150, 172], [0, 0], 18, 12, 2.0, "man", "z")
    h = rad.ObjCnt([a, b, c, coil])
    r2 = np.random.default_rng(23)
    P = np.column_stack([r2.uniform(-150, 150, 300), r2.uniform(-150, 150, 300),
                         r2.uniform(-45, 45, 300)]) + 0.0371
    return _solve_pair(rad, h, P.tolist(), 9, 1e-9, 5000)


def case_single_precision_field(rad):
    h = MD.mixed_sym(rad)
    P = GOLD["cases"]["mixed_sym"]["points"]
    rad.Solve(h, 1e-8, 3000, 4)
    out = {"b_f32": rad.Fld(h, "b", P, use_gpu=True, precision="single"), "fld_f32": rad.UtiFldLastBackend(),
           "b_cpu": rad.Fld(h, "b", P, use_gpu=False)}
    return out


def case_srcobj(rad):
    """A frozen magnet array as the extra source of a relaxed iron block
    (RlxPre srcobj): its field at the block's elements is evaluated by the
    plugin's field path (radGPU_ComputeFieldFromSrcRep)."""
    src = MD.magnet_array(rad, nside=2, div=2)
    rad.Solve(src, 1e-10, 1000, 4)
    iron = rad.ObjRecMag([0.37, -0.21, 14.1], [20, 20, 6], [0, 0, 0])
    rad.MatApl(iron, rad.MatSatIsoFrm([2000, 1.5], [100, 0.4], [10, 0.2]))
    rad.ObjDivMag(iron, [3, 3, 2])
    P = (MD.magnet_array_points(9, 4) * [0.5, 0.5, 1.0] + [0.011, 0.023, 12.0]).tolist()
    out = {}
    im = rad.RlxPre(iron, src, use_gpu=True)
    out["asm_gpu"] = rad.UtiAsmLastBackend()
    out["st_gpu"] = list(rad.RlxAuto(im, 1e-10, 3000, 9, "ZeroM->True"))
    out["b_gpu"] = rad.Fld(iron, "b", P, use_gpu=False)
    im2 = rad.RlxPre(iron, src, use_gpu=False)
    out["st_cpu"] = list(rad.RlxAuto(im2, 1e-10, 100000, 4, "ZeroM->True"))
    out["b_cpu"] = rad.Fld(iron, "b", P, use_gpu=False)
    return out


def case_cpu_assembly_gpu_relax(rad):
    """Matrix assembled by the core's CPU loop, relaxed on the device (the
    matrix is loaded from the core's host copy)."""
    h = MD.magnet_array(rad, nside=2, div=2)
    P = MD.magnet_array_points(7, 5).tolist()
    im = rad.RlxPre(h, use_gpu=False)
    out = {"asm": rad.UtiAsmLastBackend(), "st_gpu": list(rad.RlxAuto(im, 1e-11, 2000, 9, "ZeroM->True"))}
    out["b_gpu"] = rad.Fld(h, "b", P, use_gpu=False)
    out["st_cpu"] = list(rad.RlxAuto(im, 1e-11, 100000, 4, "ZeroM->True"))
    out["b_cpu"] = rad.Fld(h, "b", P, use_gpu=False)
    return out


def case_material_change(rad):
    """MatApl between RlxPre and RlxAuto: the next relaxation uses the new law
    on both paths."""
    h = MD.magnet_array(rad, nside=2, div=2)
    P = MD.magnet_array_points(7, 5).tolist()
    im = rad.RlxPre(h, use_gpu=True)
    rad.RlxAuto(im, 1e-11, 2000, 9)
    rad.MatApl(h, rad.MatLin([0.3, 0.4], [0.0, 0.0, 1.0]))
    out = {"st_gpu": list(rad.RlxAuto(im, 1e-11, 2000, 9, "ZeroM->True"))}
    out["b_gpu"] = rad.Fld(h, "b", P, use_gpu=False)
    out["st_cpu"] = list(rad.RlxAuto(im, 1e-11, 100000, 4, "ZeroM->True"))
    out["b_cpu"] = rad.Fld(h, "b", P, use_gpu=False)
    return out


def case_direct_solve(rad):
    """Linear tetrahedral mesh (chi = 5): the device direct solve (FP64 and
    TF32 + GMRES-IR) against the CPU relaxation of the same interaction."""
    c = GOLD["cases"]["tet_mesh_150"]
    h = MD.tet_mesh(rad, **c["kwargs"])
    h = h[0] if isinstance(h, tuple) else h
    P = c["points"]
    im = rad.RlxPre(h, use_gpu=True)
    out = {"asm_gpu": rad.UtiAsmLastBackend()}
    out["st_f64"] = refmodule.direct_solve(im, "f64").tolist()
    out["b_f64"] = rad.Fld(h, "b", P, use_gpu=True)
    out["st_tf32"] = refmodule.direct_solve(im, "tf32").tolist()
    out["b_tf32"] = rad.Fld(h, "b", P, use_gpu=True)
    out["st_cpu"] = list(rad.RlxAuto(im, 1e-12, 200000, 4, "ZeroM->True"))
    out["b_cpu"] = rad.Fld(h, "b", P, use_gpu=False)
    return out


# A soft-iron curve |M|(mu0 |H|) in T, tabulated (the shape of a low-carbon
# steel: steep start, knee near 1.4 T, saturation near 2.1 T)
IRON_TABLE = [[0.0, 0.0], [1e-4, 0.28], [3e-4, 0.72], [6e-4, 1.05], [1e-3, 1.25], [2e-3, 1.45],
              [4e-3, 1.58], [8e-3, 1.70], [2e-2, 1.83], [5e-2, 1.93], [0.1, 2.0], [0.3, 2.07],
              [1.0, 2.12], [3.0, 2.15]]


def _table_yoke(rad):
    rad.UtiDelAll()
    rad.FldLenRndSw("off")
    pieces = []
    for c, d, k in (([15.0, 0.0, 30.0], [30.0, 40.0, 20.0], [3, 2, 2]), ([45.0, 0.0, 47.5], [90.0, 40.0, 15.0], [4, 2, 1]),
                    ([80.0, 0.0, 20.37], [20.0, 40.0, 40.0], [2, 2, 3])):
        b = rad.ObjRecMag(c, d, [0, 0, 0])
        rad.ObjDivMag(b, k)
        pieces.append(b)
    yoke = rad.ObjCnt(pieces)
    rad.MatApl(yoke, rad.MatSatIsoTab(IRON_TABLE))
    rad.TrfZerPerp(yoke, [0, 0, 0], [1, 0, 0])
    rad.TrfZerPara(yoke, [0, 0, 0], [0, 0, 1])
    coil = rad.ObjRaceTrk([0, 0, 30], [2, 14], [40, 50], 16, 6, 25.0, "man", "z")
    h = rad.ObjCnt([yoke, coil])
    P = MD.iron_dipole_points(5, 30.0)
    return h, P.tolist()


def case_table_m9(rad):
    """Tabulated M(H) (MatSatIsoTab) relaxed by method 9 on the device."""
    h, P = _table_yoke(rad)
    return _solve_pair(rad, h, P, 9, 1e-10, 5000)


def case_table_m11(rad):
    h, P = _table_yoke(rad)
    return _solve_pair(rad, h, P, 11, 1e-10, 5000)


def case_break_policy(rad):
    """UtiGpuFallback('break'): an assembly the GPU cannot take raises
    Radia::Error602 instead of falling back (used where no device exists)."""
    h = MD.magnet_array(rad, nside=2, div=1)
    prev = rad.UtiGpuFallback()
    rad.UtiGpuFallback("break")
    try:
        rad.RlxPre(h, use_gpu=True)
        raised = ""
    except RuntimeError as e:
        raised = str(e)
    finally:
        rad.UtiGpuFallback(prev)
    im = rad.RlxPre(h, use_gpu=True)
    return {"raised": raised, "asm": rad.UtiAsmLastBackend(), "policy": prev,
            "st": list(rad.RlxAuto(im, 1e-10, 1000, 9))}


def main(names):
    rad = refmodule.load()
    res = {}
    for n in names:
        res[n] = globals()["case_" + n](rad)
    print("SHIM_JSON " + json.dumps(res))


if __name__ == "__main__":
    main(sys.argv[1:])
