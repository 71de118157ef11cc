"""CUDA path (libradb200 through the C-ABI) against the CPU oracle and the
reference's golden vectors.

Tolerances: fields of given magnetization 1e-10 relative in FP64 (the
reference's GPU-vs-CPU bar is 1e-9, tests/test_gpu_fld_fp32.py:71 of the
reference), FP32 field option 5e-4 (same file, :72); FP64 interaction matrix
1e-12 relative to the oracle's FP64 assembly; relaxed models 5e-6 (linear) /
5e-5 (saturating) relative in B, as the reference's tests/test_recmag_asm.py.
"""
import json
import os

import numpy as np
import pytest

import models as MD
from radiacuda_b200 import _native, model
from util import leaf_magnetizations, rel_err

import oracle.oracle as O

pytestmark = pytest.mark.gpu

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


def _randomize_m(rad, h, seed=0):
    rng = np.random.default_rng(seed)
    for lf in model.collect_leaves(rad._objs, h):
        if hasattr(lf.obj, "m") and not (hasattr(lf.obj, "j") and np.any(lf.obj.j != 0)):
            lf.obj.m = rng.normal(size=3)


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_field_fp64_matches_oracle(cuda, rad, name):
    h, c = _build(rad, name)
    _randomize_m(rad, h)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    P = np.array(c["points"])
    for what in (0, 1, 2):
        got = _native.field(g, P, what, 0)
        exp = O.field(g, P, what)
        if what == 2:
            assert np.array_equal(got, exp)
        else:
            assert rel_err(got, exp) < 1e-10


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_field_golden_before_relaxation(cuda, rad, name):
    h, c = _build(rad, name)
    B = np.array(rad.Fld(h, "b", c["points"]))
    assert rel_err(B, np.array(c["b_before"])) < 1e-9
    assert rad.UtiFldLastBackend() == "gpu"


def test_field_fp32_option(cuda, rad):
    h, c = _build(rad, "tet_mesh_150")
    _randomize_m(rad, h, 1)
    P = np.array(c["points"])
    b64 = np.array(rad.Fld(h, "b", P.tolist()))
    b32 = np.array(rad.Fld(h, "b", P.tolist(), precision="single"))
    assert rel_err(b32, b64) < 5e-4
    h, c = _build(rad, "magnet_array_2x2")
    P = np.array(c["points"])
    assert rel_err(np.array(rad.Fld(h, "b", P.tolist(), precision="single")), np.array(rad.Fld(h, "b", P.tolist()))) < 5e-4


def test_field_is_bitwise_reproducible_and_chunk_invariant(cuda, rad):
    h, c = _build(rad, "mixed_sym")
    _randomize_m(rad, h, 2)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    P = np.random.default_rng(4).uniform(-90, 90, size=(5000, 3))
    a = _native.field(g, P, 0)
    b = _native.field(g, P, 0)
    assert np.array_equal(a, b)
    # a subset evaluated alone (different source chunking) agrees to rounding
    s = _native.field(g, P[:37], 0)
    assert rel_err(s, a[:37]) < 1e-13


def test_field_empty_and_single_point(cuda, rad):
    h, c = _build(rad, "magnet_array_2x2")
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    assert _native.field(g, np.zeros((0, 3)), 0).shape == (0, 3)
    one = _native.field(g, np.array([[0.31, 0.27, 17.3]]), 0)
    assert rel_err(one, O.field(g, np.array([[0.31, 0.27, 17.3]]), 0)) < 1e-12


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_assembly_fp64_matches_oracle(cuda, rad, name):
    h, c = _build(rad, name)
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    nat = _native.NativeInteraction(pack, 1)
    try:
        N = nat.matrix(np.float64)
        Hx = nat.extfield()
    finally:
        nat.free()
    No = O.assemble(pack)
    assert np.all(np.isfinite(N))
    assert np.abs(N - No).max() <= 1e-12 * np.abs(No).max()
    Ho = O.extfield(pack)
    assert np.abs(Hx - Ho).max() <= 1e-12 * max(np.abs(Ho).max(), 1e-300)


def test_assembly_fp32_is_rounded_fp64(cuda, rad):
    h, c = _build(rad, "tet_mesh_150")
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    nat = _native.NativeInteraction(pack, 0)
    try:
        N32 = nat.matrix(np.float32)
    finally:
        nat.free()
    No = O.assemble(pack).astype(np.float32)
    ulp = np.spacing(np.abs(No))
    assert np.all(np.abs(N32 - No) <= ulp)


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_solve_matches_reference_golden(cuda, rad, name):
    h, c = _build(rad, name)
    st = rad.Solve(h, c["prec"], 5000, 4)
    assert st[0] <= c["prec"]
    tol = 5e-6 if name in LINEAR else 5e-5
    B = np.array(rad.Fld(h, "b", c["points"]))
    assert rel_err(B, np.array(c["b"])) < tol
    Mo = leaf_magnetizations(rad, h)
    assert rel_err(Mo, np.array(c["M"])) < (1e-6 if name in LINEAR else 1e-4)


@pytest.mark.parametrize("name", ["mixed_sym", "iron_dipole_300"])
def test_newton_krylov_matches_reference_golden(cuda, rad, name):
    h, c = _build(rad, name)
    im = rad.RlxPre(h)
    st = rad.RlxAuto(im, c["prec"], 2000, 11)
    assert st[0] <= c["prec"]
    B = np.array(rad.Fld(h, "b", c["points"]))
    assert rel_err(B, np.array(c["b"])) < 5e-5


@pytest.mark.parametrize("kind", ["small", "mixed"])
def test_reference_mpi_solve_golden_on_gpu(cuda, rad, kind):
    h = MD.mpi_solve_model(rad, kind)
    rad.Solve(h, 1e-5, 3000, 4)
    b = np.array(rad.Fld(h, "b", GOLD["mpi_solve_points"]))
    assert rel_err(b, np.array(GOLD["mpi_solve"][kind]["b"])) < 1e-5


@pytest.mark.parametrize("name", ["magnet_array_2x2", "tet_mesh_150", "sym_blocks"])
@pytest.mark.parametrize("meth", [12, 13])
def test_direct_solve_matches_fp64_oracle(cuda, rad, name, meth):
    h, c = _build(rad, name)
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    Md = O.linear_direct(pack, O.assemble(pack), O.extfield(pack))
    im = rad.RlxPre(h, storage="f64")
    st = rad.RlxAuto(im, 1e-10, 200, meth)
    M = rad._objs[im].M
    assert rel_err(M, Md) < 1e-9
    rad.UtiDel(im)


def test_kernel_launch_counter_advances(cuda, rad):
    before = _native.kernel_launches()
    h, c = _build(rad, "magnet_array_2x2")
    rad.Fld(h, "b", c["points"])
    assert _native.kernel_launches() > before


# ---------------------------------------------------------------------------
# vertex/edge polyhedron form (fast path): same exact field, fewer transcendentals
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["tet_mesh_150", "mixed_sym"])
def test_fast_polyhedron_field_matches_oracle(cuda, rad, name):
    h, c = _build(rad, name)
    _randomize_m(rad, h, 3)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    P = np.array(c["points"])
    for what in (0, 1, 2):
        got = _native.field(g, P, what, 2)
        exp = O.field(g, P, what)
        if what == 2:
            assert np.array_equal(got, exp)
        else:
            assert rel_err(got, exp) < 1e-10


def test_fast_polyhedron_fp32_field(cuda, rad):
    h, c = _build(rad, "tet_mesh_150")
    _randomize_m(rad, h, 4)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    P = np.array(c["points"])
    assert rel_err(_native.field(g, P, 0, 1), O.field(g, P, 0)) < 5e-5


@pytest.mark.parametrize("name", ["tet_mesh_150", "mixed_sym"])
def test_fast_polyhedron_assembly_matches_oracle(cuda, rad, name):
    h, c = _build(rad, name)
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    nat = _native.NativeInteraction(pack, 1 | 16)
    try:
        N = nat.matrix(np.float64)
    finally:
        nat.free()
    No = O.assemble(pack)
    assert np.abs(N - No).max() <= 1e-10 * np.abs(No).max()
