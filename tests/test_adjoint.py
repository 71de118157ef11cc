"""Adjoint of the relaxation and of the field operator.

CPU tests pin the oracle's restatement of the adjoint (oracle/adjoint_oracle.py)
to FP64 central finite differences of the oracle's own forward problem
(assembly + solve + field).  GPU tests compare the device adjoint
(radb200_adjoint_solve / adjoint_grad / field_vjp through the C-ABI) with the
oracle's, element by element, and spot-check it against central differences
of the device forward solve.

Loss: L = sum_k W_k . B(x_k) with fixed random weights W (dL/dB = W), so the
gradient is exactly what the adjoint contracts.
"""
import copy

import numpy as np
import pytest

import models as MD
from oracle import adjoint_oracle as AO
from oracle import oracle as O
from radiacuda_b200 import model

H_FD = 1e-5          # central-difference step (mm for centres/widths, T for Mr)
TOL_FD = 1e-6        # |adjoint - FD| / max |gradient|
TOL_DEVICE = 1e-8    # device adjoint vs oracle adjoint, / max |gradient|


def _pack(rad, h):
    return model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))


def oracle_forward(pack, pts, W):
    N = O.assemble(pack)
    Hext = O.extfield(pack)
    if np.all(pack.mat_kind == 0):
        M = O.linear_direct(pack, N, Hext)
    else:
        M = AO.solve_newton(pack, N, Hext)
    return M, float(np.sum(AO.field_of(pack, M, pts, 0) * W))


def perturbed(pack, which, e, a, h):
    p = copy.deepcopy(pack)
    kind, idx = p.elem_src[e]
    if which == "c":
        p.elems["rec"][idx, a] += h
    elif which == "d":
        p.elems["rec"][idx, 3 + a] += h
    elif which == "Mr":
        p.mat[e, 9 + a] += h
    elif which == "chi":
        p.mat[e, a] += h
    return p


def fd_grad(pack, pts, W, which, e, a, h=H_FD):
    _, lp = oracle_forward(perturbed(pack, which, e, a, h), pts, W)
    _, lm = oracle_forward(perturbed(pack, which, e, a, -h), pts, W)
    return (lp - lm) / (2 * h)


def linear_case(rad):
    h = MD.adjoint_linear(rad)
    pack = _pack(rad, h)
    pts = MD.adjoint_points()
    W = np.random.default_rng(5).normal(size=pts.shape)
    return pack, pts, W


def nonlinear_case(rad):
    h, _, _, _ = MD.hybrid_undulator(rad, n_pairs=2, pole_div=(2, 1, 2), block_div=(2, 1, 1))
    pack = _pack(rad, h)
    pts = MD.hybrid_points(n=120, n_pairs=2)
    W = np.random.default_rng(6).normal(size=pts.shape)
    return pack, pts, W


# ---------------------------------------------------------------------------
# CPU: the analytic cuboid-tensor derivative and the oracle adjoint
# ---------------------------------------------------------------------------
def _unit_Q(rad, c, d, x):
    Q = np.zeros((3, 3))
    for a in range(3):
        MD.reset(rad)
        m = np.zeros(3)
        m[a] = 1.0
        h = rad.ObjRecMag(list(c), list(d), list(m))
        Q[:, a] = O.field(model.pack_sources(rad._objs, h, (0, 0, 0)), np.array([x]), 1)[0]
    return Q


@pytest.mark.parametrize("x", [[5.3, 4.1, -3.7], [-1.2, -6.5, 2.9], [1.3, -2.4, 0.8]])
def test_cuboid_tensor_derivative_matches_oracle_fd(rad, x):
    c, d = np.array([1.0, -2.0, 0.5]), np.array([4.0, 3.0, 2.5])
    x = np.array(x)
    dQq, dQh = AO.cuboid_dQ(x - c, 0.5 * d)
    h = 1e-5
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        fq = (_unit_Q(rad, c, d, x + e) - _unit_Q(rad, c, d, x - e)) / (2 * h)
        fh = (_unit_Q(rad, c, d + 2 * e, x) - _unit_Q(rad, c, d - 2 * e, x)) / (2 * h)
        assert np.abs(fq - dQq[..., k]).max() < 1e-7 * max(1.0, np.abs(dQq).max())
        assert np.abs(fh - dQh[..., k]).max() < 1e-7 * max(1.0, np.abs(dQh).max())


@pytest.mark.parametrize("case", ["linear", "nonlinear"])
def test_oracle_adjoint_matches_central_differences(rad, case):
    pack, pts, W = linear_case(rad) if case == "linear" else nonlinear_case(rad)
    M, _ = oracle_forward(pack, pts, W)
    g = AO.gradients(pack, M, pts, W)
    n = pack.elem_src.shape[0]
    rng = np.random.default_rng(7)
    checks = [("c", e, a) for e in rng.choice(n, 4, replace=False) for a in range(3)]
    checks += [("d", e, a) for e in rng.choice(n, 3, replace=False) for a in range(3)]
    lin = [e for e in range(n) if pack.mat_kind[e] == 0]
    checks += [("Mr", e, a) for e in rng.choice(lin, 2, replace=False) for a in range(3)]
    checks += [("chi", int(rng.choice(lin)), a) for a in (0, 4, 5)]
    scale = {k: np.abs(g[k]).max() for k in ("c", "d", "Mr", "chi")}
    for which, e, a in checks:
        fd = fd_grad(pack, pts, W, which, int(e), a)
        got = g[which][(9 if which == "chi" else 3) * int(e) + a]
        assert abs(got - fd) <= TOL_FD * scale[which] + 1e-12, (which, e, a, got, fd)


# ---------------------------------------------------------------------------
# GPU: the device adjoint against the oracle's
# ---------------------------------------------------------------------------
def device_forward(pack, storage, nonlinear):
    from radiacuda_b200 import _native
    I = _native.NativeInteraction(pack, storage=storage)
    if nonlinear:
        M, _, st = I.relax(1, 1e-13, 200, True, 1.0, np.zeros(3 * pack.elem_src.shape[0]))
    else:
        M, st = I.direct(0, 1e-13, 50)
    return I, M


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["linear", "nonlinear"])
def test_device_adjoint_matches_oracle(cuda, rad, case):
    pack, pts, W = linear_case(rad) if case == "linear" else nonlinear_case(rad)
    I, M = device_forward(pack, 1, case == "nonlinear")
    ref = AO.gradients(pack, M, pts, W)
    gM, gc_f, gd_f = I.field_vjp(M, pts, 0, W)
    assert np.abs(gM - ref["gM"]).max() <= TOL_DEVICE * np.abs(ref["gM"]).max()
    lam, st = I.adjoint_solve(gM, 1e-13, 300)
    assert st[0] <= 1e-13
    assert np.abs(lam - ref["lam"]).max() <= TOL_DEVICE * np.abs(ref["lam"]).max()
    g = I.adjoint_grad(lam)
    got = dict(Mr=g["Mr"], chi=g["chi"], c=g["c"] + gc_f, d=g["d"] + gd_f)
    for k in ("Mr", "chi", "c", "d"):
        assert np.abs(got[k] - ref[k]).max() <= TOL_DEVICE * max(np.abs(ref[k]).max(), 1e-30), k


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [0, 2])
def test_device_adjoint_through_lu_factors(cuda, rad, storage):
    """Linear model solved by the direct solver (FP64 LU, or TF32 LU with FP64
    refinement on mixed storage): the adjoint reuses the kept factors."""
    from radiacuda_b200 import _native
    pack, pts, W = linear_case(rad)
    I = _native.NativeInteraction(pack, storage=storage)
    M, st = I.direct(0 if storage == 0 else 1, 1e-13, 60)
    ref = AO.gradients(pack, M, pts, W)
    gM, gc_f, gd_f = I.field_vjp(M, pts, 0, W)
    lam, st = I.adjoint_solve(gM, 1e-12, 100)
    assert st[2] == 1.0  # the LU path was used
    # FP32 storage: the matrix itself is rounded, so compare at FP32 level
    tol = 1e-5 if storage == 0 else TOL_DEVICE
    assert np.abs(lam - ref["lam"]).max() <= tol * np.abs(ref["lam"]).max()
    g = I.adjoint_grad(lam)
    assert np.abs(g["c"] + gc_f - ref["c"]).max() <= tol * np.abs(ref["c"]).max()


@pytest.mark.gpu
def test_autograd_undulator_block_gradients_match_central_differences(cuda, rad):
    """Shimming-style loss on a small planar undulator: block remanence vectors
    (with the easy-axis susceptibility chi(Mr)) and block-centre offsets, through
    torch autograd, against central differences of the device forward solve
    (steps 1e-6 T and 1e-6 mm as the workload specifies)."""
    import torch

    from radiacuda_b200 import adjoint as A

    nper = 4
    h, blocks = MD.undulator(rad, nper_row=nper, div=2)
    pts = MD.undulator_points(n=400, nper_row=nper)
    prob = A.FieldProblem(h, pts, "b")
    ksi = prob.linear_ksi()
    blk_of = np.zeros(prob.n, dtype=np.int64)
    for b, hb in enumerate(blocks):
        blk_of[prob.elements_of(hb)] = b
    nb = len(blocks)
    mr_blk0 = np.array([prob.mr0[blk_of == b][0] for b in range(nb)])
    z = torch.tensor(pts[:, 2])
    target = 0.8 * torch.sin(2 * np.pi * z / 20.0)

    def loss_of(mr_blk, dc_blk):
        mr = mr_blk[torch.as_tensor(blk_of)]
        chi = A.FieldProblem.aniso_chi(mr, ksi)
        centre = torch.as_tensor(prob.centre0) + dc_blk[torch.as_tensor(blk_of)]
        B = A.relaxed_field(prob, mr, chi, centre, torch.as_tensor(prob.dims0))
        return torch.sum((B[:, 1] - target) ** 2)

    mr_blk = torch.tensor(mr_blk0, requires_grad=True)
    dc_blk = torch.zeros((nb, 3), dtype=torch.float64, requires_grad=True)
    L = loss_of(mr_blk, dc_blk)
    L.backward()
    st = prob.last_status["adjoint"]
    assert st[0] <= 1e-12
    rng = np.random.default_rng(3)
    for b in rng.choice(nb, 3, replace=False):
        for a in range(3):
            for which in ("mr", "dc"):
                hstep = 1e-6
                vals = []
                for s in (1, -1):
                    m = torch.tensor(mr_blk0)
                    d = torch.zeros((nb, 3), dtype=torch.float64)
                    (m if which == "mr" else d)[b, a] += s * hstep
                    with torch.no_grad():
                        vals.append(float(loss_of(m, d)))
                fd = (vals[0] - vals[1]) / (2 * hstep)
                got = float((mr_blk.grad if which == "mr" else dc_blk.grad)[b, a])
                scale = float((mr_blk.grad if which == "mr" else dc_blk.grad).abs().max())
                assert abs(got - fd) <= 1e-5 * scale, (which, b, a, got, fd)


# ---------------------------------------------------------------------------
# pinned to the reference: finite differences of the reference CPU Radia
# (tests/golden/adjoint_fd.json, made by tests/golden/make_adjoint_golden.py)
# ---------------------------------------------------------------------------
def _golden_fd():
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "adjoint_fd.json")) as f:
        return json.load(f)


def block_gradients(pack, blocks, rad, g):
    """Per-block d/dMr (through M and the easy-axis chi(Mr), radmater.h:292-303)
    and d/dcentre from per-element gradients g (dict Mr, chi, c)."""
    leaf_block = {}
    for b, hb in enumerate(blocks):
        for lf in model.collect_leaves(rad._objs, hb):
            leaf_block[lf.handle] = b
    nb = len(blocks)
    gmr, gc = np.zeros((nb, 3)), np.zeros((nb, 3))
    for e, lf in enumerate(pack.leaves):
        b = leaf_block[lf.handle]
        mr = pack.mat[e, 9:12]
        kpar, kperp = lf.obj.mat.ksi
        amr = np.linalg.norm(mr)
        L = mr / amr
        dL = (np.eye(3) - np.outer(L, L)) / amr  # column a: dL/dmr_a
        gchi = g["chi"][9 * e:9 * e + 9].reshape(3, 3)
        for a in range(3):
            dchi = (kpar - kperp) * (np.outer(dL[:, a], L) + np.outer(L, dL[:, a]))
            gmr[b, a] += g["Mr"][3 * e + a] + np.sum(gchi * dchi)
        gc[b] += g["c"][3 * e:3 * e + 3]
    return gmr, gc


def _check_against_golden(G, gmr, gc):
    for kind, got in (("mr", gmr), ("c", gc)):
        ref = G["grad_" + kind]
        scale = max(abs(v) for v in ref.values())
        for key, v in ref.items():
            b, a = map(int, key.split(","))
            assert abs(got[b, a] - v) <= 5e-5 * scale, (kind, key, got[b, a], v)


def test_oracle_adjoint_matches_reference_finite_differences(rad):
    G = _golden_fd()
    h, blocks = MD.undulator(rad, nper_row=G["nper_row"], div=G["div"])
    pack = _pack(rad, h)
    pts = MD.undulator_points(n=G["n_points"], nper_row=G["nper_row"])
    W = np.random.default_rng(G["w_seed"]).normal(size=pts.shape)
    M, L = oracle_forward(pack, pts, W)
    assert abs(L - G["loss"]) <= 1e-6 * abs(G["loss"])
    _check_against_golden(G, *block_gradients(pack, blocks, rad, AO.gradients(pack, M, pts, W)))


@pytest.mark.gpu
def test_device_adjoint_matches_reference_finite_differences(cuda, rad):
    from radiacuda_b200 import adjoint as A
    G = _golden_fd()
    h, blocks = MD.undulator(rad, nper_row=G["nper_row"], div=G["div"])
    pts = MD.undulator_points(n=G["n_points"], nper_row=G["nper_row"])
    W = np.random.default_rng(G["w_seed"]).normal(size=pts.shape)
    prob = A.FieldProblem(h, pts, "b")
    L = float(np.sum(prob.forward() * W))
    assert abs(L - G["loss"]) <= 1e-6 * abs(G["loss"])
    g = prob.backward(W)
    ge = dict(Mr=g["mr"].reshape(-1), chi=g["chi"].reshape(-1), c=g["centre"].reshape(-1))
    _check_against_golden(G, *block_gradients(prob.pack, blocks, rad, ge))
