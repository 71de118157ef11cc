"""The CPU oracle (oracle/radia_oracle.c) against the reference's own numbers.

Pins the restatement before anything is compared with it:
  * the known answer of the reference's first example;
  * golden fields / relaxed magnetizations produced by the reference CPU module
    (tests/golden/golden.json, made by tests/golden/make_golden.py);
  * the golden B values of the reference's MPI-solve regression;
  * live comparisons with the compiled reference module when it is present.
Tolerances follow the reference's own parity tests: 1e-9 relative for fields
of given magnetizations (tests/test_gpu_fld_fp32.py of the reference), 5e-6 /
5e-5 relative for linear / saturating relaxed models (tests/test_recmag_asm.py).
"""
import json
import os

import numpy as np
import pytest

import models as MD
from radiacuda_b200 import model
from util import leaf_magnetizations, rel_err

import oracle.oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))

BUILDERS = {
    "magnet_array_2x2": MD.magnet_array,
    "sym_blocks": MD.sym_blocks,
    "mixed_sym": MD.mixed_sym,
    "iron_dipole_300": MD.iron_dipole,
    "tet_mesh_150": MD.tet_mesh,
    "thckpgn_4": MD.thckpgn_model,
}
LINEAR = {"magnet_array_2x2", "sym_blocks", "tet_mesh_150"}


def _build(rad, name):
    c = GOLD["cases"][name]
    res = BUILDERS[name](rad, **c["kwargs"])
    return (res[0] if isinstance(res, tuple) else res), c


def oracle_solve(rad, h, prec, max_iter):
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    N = O.assemble(pack)
    H = O.extfield(pack)
    M, _, st = O.relax_m4(pack, N.astype(np.float32), H, prec, max_iter)
    for e, lf in enumerate(pack.leaves):
        lf.obj.m = M[3 * e:3 * e + 3].copy()
    return pack, M, st


def test_example01_known_answer(rad):
    rad.UtiDelAll()
    rad.FldLenRndSw("off")
    m = rad.ObjRecMag([0, 0, 0], [1, 1, 1], [-0.5, 1, 0.7])
    b = O.field(model.pack_sources(rad._objs, m, tuple(rad._rand)), [[0.52, 0.6, 0.7]], 0)[0]
    assert rel_err(b, GOLD["example01"]["b"]) < 1e-13
    assert np.allclose(b, GOLD["example01"]["expected_approx"], rtol=1e-4)


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_field_of_given_magnetization(rad, name):
    h, c = _build(rad, name)
    P = np.array(c["points"])
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    assert rel_err(O.field(g, P, 0), np.array(c["b_before"])) < 1e-9


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_relaxation_matches_reference(rad, name):
    h, c = _build(rad, name)
    pack, M, st = oracle_solve(rad, h, c["prec"], 5000)
    tol = 5e-6 if name in LINEAR else 5e-5
    P = np.array(c["points"])
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    assert rel_err(O.field(g, P, 0), np.array(c["b"])) < tol
    assert rel_err(O.field(g, P, 1), np.array(c["h"])) < tol
    Mg = np.array(c["M"])
    Mo = leaf_magnetizations(rad, h)      # lab frame, every symmetry image
    assert Mg.shape == Mo.shape
    assert rel_err(Mo, Mg) < (1e-6 if name in LINEAR else 1e-4)


@pytest.mark.parametrize("kind", ["small", "mixed"])
def test_reference_mpi_solve_golden(rad, kind):
    h = MD.mpi_solve_model(rad, kind)
    oracle_solve(rad, h, 1e-5, 3000)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    b = O.field(g, np.array(GOLD["mpi_solve_points"]), 0)
    assert rel_err(b, np.array(GOLD["mpi_solve"][kind]["b"])) < 1e-6


def test_linear_direct_is_the_relaxation_fixed_point(rad):
    h, c = _build(rad, "magnet_array_2x2")
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    N = O.assemble(pack)
    H = O.extfield(pack)
    Md = O.linear_direct(pack, N, H)
    Mi, _, _ = O.relax_m4(pack, N, H, 1e-13, 500)
    assert rel_err(Mi, Md) < 1e-11


def test_live_reference_random_sources(ref, rad):
    """Random cuboids / tetrahedra / arcs with random M: oracle == reference."""
    rng = np.random.default_rng(5)
    worst = 0.0
    for trial in range(6):
        hs = {}
        for R, key in ((ref, "ref"), (rad, "ours")):
            R.UtiDelAll()
            R.FldLenRndSw("off")
        r2 = np.random.default_rng(100 + trial)
        c = r2.uniform(-10, 10, 3)
        d = r2.uniform(1, 6, 3)
        m = r2.normal(size=3)
        v = r2.uniform(0, 5, (4, 3)) + r2.uniform(-10, 10, 3)
        for R, key in ((ref, "ref"), (rad, "ours")):
            a = R.ObjRecMag(c.tolist(), d.tolist(), m.tolist())
            t = R.ObjPolyhdr(v.tolist(), MD.TET_FACES, (m[::-1]).tolist())
            arc = R.ObjArcCur([1, 2, 3], [3, 5], [0.2, 2.5], 4, 7, 2.5, "man", "y")
            hs[key] = R.ObjCnt([a, t, arc])
        P = rng.uniform(-25, 25, size=(40, 3))
        br = np.array(ref.Fld(hs["ref"], "b", P.tolist()))
        bo = O.field(model.pack_sources(rad._objs, hs["ours"], tuple(rad._rand)), P, 0)
        worst = max(worst, rel_err(bo, br))
    assert worst < 1e-11
