"""Parity on the five benchmark configurations at their stated sizes, against
fields of the reference Radia CPU module (tests/golden/baseline_configs.npz,
made by tests/golden/make_baseline_golden.py).

Tolerances, per point (|dB_i| / |B_i|, points where |B_i| is below 1e-3 of
the largest measured against that floor) and as the max-norm ratio: 5e-6 for
linear and 5e-5 for saturating materials after relaxation (the reference's
tests/test_recmag_asm.py:134-157 bars); 1e-6 for the 3,000-tetrahedron
chi = 1000 direct solve against the FP64 oracle (c3o: the CPU oracle's
interaction matrix, LAPACK, the oracle's field) -- the precision target, for
the plain FP64 path and for the mixed path (TF32 tensor-core LU + FP64
GMRES-IR, FP32 field terms). Against the system built from the reference's
own element fields (c3) the bar is 5e-6: one of its 3,000 self blocks is off
by 1e-4 (a tolerance branch of the reference's polygon integrals on a nearly
axis-parallel edge; tests/test_oracle_quadrature.py shows the oracle right
there against an independent quadrature), and at chi = 1000 that element
alone moves B outside by 3.0e-6, the gap between the two goldens.
"""
import os

import numpy as np
import pytest

import models as MD

pytestmark = pytest.mark.gpu

GOLD_PATH = os.path.join(os.path.dirname(__file__), "golden", "baseline_configs.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD_PATH))


def errs(got, exp):
    g = np.asarray(got, dtype=float).reshape(-1, 3)
    e = np.asarray(exp, dtype=float).reshape(-1, 3)
    d = np.linalg.norm(g - e, axis=1)
    n = np.linalg.norm(e, axis=1)
    return float(np.abs(g - e).max() / np.abs(e).max()), float((d / np.maximum(n, 1e-3 * n.max())).max())


def _relaxed_field(rad, model, P, prec, iters):
    st = rad.Solve(model, prec, iters, 4)
    assert st[0] <= prec, st
    return np.array(rad.Fld(model, "b", P.tolist()))


def test_c1_magnet_array_432(cuda, rad, gold):
    h = MD.magnet_array(rad)
    B = _relaxed_field(rad, h, MD.magnet_array_points(), 1e-10, 10000)
    e = errs(B, gold["c1_b"])
    assert e[0] < 5e-6 and e[1] < 5e-6, e


def test_c2_iron_dipole_4000_four_images_racetrack(cuda, rad, gold):
    h = MD.iron_dipole(rad, n_target=4000)
    P = MD.iron_dipole_points(100)[gold["c2_idx"]]
    B = _relaxed_field(rad, h, P, 1e-9, 20000)
    e = errs(B, gold["c2_b"])
    assert gold["c2_status"][0] < 2e-7
    assert e[0] < 5e-5 and e[1] < 5e-5, e


def test_c4_planar_undulator_640(cuda, rad, gold):
    h, _ = MD.undulator(rad)
    B = _relaxed_field(rad, h, MD.undulator_points(), 1e-10, 10000)
    e = errs(B, gold["c4_b"])
    assert e[0] < 5e-6 and e[1] < 5e-6, e


def test_c5_hybrid_undulator_6080(cuda, rad, gold):
    h = MD.hybrid_undulator(rad)[0]
    P = MD.hybrid_points()[gold["c5_idx"]]
    B = _relaxed_field(rad, h, P, 1e-9, 20000)
    e = errs(B, gold["c5_b"])
    assert gold["c5_status"][0] < 2e-7
    assert e[0] < 5e-5 and e[1] < 5e-5, e


@pytest.mark.parametrize("path", ["plain_f64", "mixed"])
def test_c3_chi1000_direct_solve_3000_tets_vs_fp64_oracle(cuda, rad, gold, path):
    whole, body = MD.tet_mesh(rad, ncell=8, n_tets=3000, chi=1000.0)
    P = MD.tet_mesh_points(2000, ncell=8)
    if path == "plain_f64":
        im = rad.RlxPre(whole, storage="f64")
        st = rad.RlxAuto(im, 1e-13, 200, 12)
        B = np.array(rad.Fld(whole, "b", P.tolist(), precision="double"))
    else:
        im = rad.RlxPre(whole, storage="mixed", fast=True)
        st = rad.RlxAuto(im, 1e-13, 200, 13)
        B = np.array(rad.Fld(whole, "b", P.tolist(), precision="single"))
    assert st[0] < 1e-12, st
    e = errs(B, gold["c3o_b"])
    assert e[0] < 1e-6 and e[1] < 1e-6, (path, e)
    g = errs(gold["c3o_b"], gold["c3_b"])
    r = errs(B, gold["c3_b"])
    assert r[0] < 5e-6 and r[1] < 5e-6, (path, r)
    # the distance to the reference-built golden is the distance between the goldens
    assert abs(r[1] - g[1]) < 0.1 * g[1], (path, r, g)
