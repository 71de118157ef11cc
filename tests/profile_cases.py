"""Small, self-contained launches of the hot kernels for profiling.

    python tests/profile_cases.py field    [--tets N] [--points P] [--precision double|single|fast]
    python tests/profile_cases.py assemble [--tets N]           (vertex/edge form, FP32 storage)
    python tests/profile_cases.py lu       [--tets N] [--mode 0|1]
    python tests/profile_cases.py relax    [--blocks N]
    python tests/profile_cases.py adjoint  [--pairs N] [--points P]

Each case builds a seeded model of the benchmark's shapes (tetrahedral mesh
of chi = 1000 material, magnet array) at a size that keeps one launch of the
kernel of interest short and the device footprint to a few GB, runs it once
and prints the wall time.  Meant to be run under ncu with -k / -c.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np


HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import models as MD  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["field", "assemble", "lu", "relax", "adjoint"])
    ap.add_argument("--pairs", type=int, default=20)
    ap.add_argument("--tets", type=int, default=20000)
    ap.add_argument("--points", type=int, default=20000)
    ap.add_argument("--blocks", type=int, default=16)
    ap.add_argument("--mode", type=int, default=1)
    ap.add_argument("--precision", default="double", choices=["double", "single", "fast"])
    a = ap.parse_args(argv)
    from radiacuda_b200 import _native, model, rad
    t0 = time.perf_counter()
    if a.case in ("field", "assemble", "lu"):
        ncell = int(np.ceil((a.tets / 6) ** (1 / 3)))
        m, body = MD.tet_mesh(rad, ncell=ncell, n_tets=a.tets)
        if a.case == "field":
            rng = np.random.default_rng(0)
            for lf in model.collect_leaves(rad._objs, body):
                lf.obj.m = rng.normal(size=3)
            P = MD.tet_mesh_points(a.points, ncell=ncell)
            t0 = time.perf_counter()
            B = rad.Fld(m, "b", P, precision=a.precision)
            print("field", P.shape[0], "points", time.perf_counter() - t0, "s", float(np.abs(B).max()))
        elif a.case == "assemble":
            im = rad.RlxPre(m, storage="f32", fast=True)
            print("assembly", time.perf_counter() - t0, "s")
        else:
            im = rad.RlxPre(m, storage="f64")
            t0 = time.perf_counter()
            st = rad.RlxAuto(im, 1e-13, 200, 12 if a.mode == 0 else 13)
            print("lu mode", a.mode, time.perf_counter() - t0, "s", st)
    elif a.case == "adjoint":
        from radiacuda_b200.adjoint import FieldProblem
        h = MD.hybrid_undulator(rad, n_pairs=a.pairs)[0]
        P = MD.hybrid_points(a.points, n_pairs=a.pairs)
        prob = FieldProblem(h, P, "b", prec=1e-12)
        prob.forward()
        t0 = time.perf_counter()
        prob.backward(np.random.default_rng(1).normal(size=P.shape))
        print("adjoint", prob.n, "elements", P.shape[0], "points", time.perf_counter() - t0, "s", prob.last_timing)
    else:
        h = MD.magnet_array(rad, nside=int(np.sqrt(a.blocks)), div=3)
        im = rad.RlxPre(h)
        t0 = time.perf_counter()
        st = rad.RlxAuto(im, 1e-10, 1000, 4)
        print("relax", time.perf_counter() - t0, "s", st)
    _native.lib().radb200_device_sync()


if __name__ == "__main__":
    main()
