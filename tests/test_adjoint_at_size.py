"""Adjoint gradients at the workload sizes, and the pole-thickness gradient
of the hybrid undulator against the reference's own finite differences.

- Pole thickness (the z width of a pole, centre fixed) enters the solve
  through the centres and widths of the pole's sub-elements: sub-element e of
  a pole of width t has centre z_e = z_pole + u_e t and width t / n_z, so
  dL/dt = sum_e (dL/dz_e) u_e + (dL/dw_e) / n_z.
- CPU: the oracle adjoint (oracle/adjoint_oracle.py) chained that way on the
  4-pair hybrid against central differences of the reference CPU module
  (tests/golden/hybrid_pole_fd.json, made by
  tests/golden/make_hybrid_adjoint_golden.py).  The reference's relaxation
  stalls near a misfit of 2e-8 on its FP32 matrix; its differences at steps
  0.02 and 0.01 mm agree to 1e-4 of the largest gradient, and the bar is
  5e-4 of it.
- GPU: the same for the device adjoint; then the 6,080-element hybrid
  (80 pairs, 4 x 4 x 4 poles) at 10,000 points, three random poles, against
  central differences of the device forward solve; and 12 random parameters
  of the 480 (80 blocks x (remanence, centre)) of the 640-element planar
  undulator at its 4,000 axis points, through torch autograd, against central
  differences with the workload's steps (1e-6 T, 1e-6 mm).
"""
import json
import os

import numpy as np
import pytest

import models as MD
from oracle import adjoint_oracle as AO
from oracle import oracle as O
from radiacuda_b200 import model


def _golden():
    with open(os.path.join(os.path.dirname(__file__), "golden", "hybrid_pole_fd.json")) as f:
        return json.load(f)


def _pole_layout(rad, pack_leaves, poles, pole_centres, pole_div):
    """Per pole: its element indices and each element's u_e."""
    out = []
    where = {lf.handle: e for e, lf in enumerate(pack_leaves)}
    for k, hp in enumerate(poles):
        es = np.array([where[lf.handle] for lf in model.collect_leaves(rad._objs, hp)], dtype=np.int64)
        cz = np.array([pack_leaves[e].obj.c[2] for e in es])
        u = (cz - pole_centres[k][2]) / MD.HYB_POLE[2]
        out.append((es, u))
    return out


def _chain(layout, gc, gd, nz):
    gc = np.asarray(gc).reshape(-1, 3)
    gd = np.asarray(gd).reshape(-1, 3)
    return np.array([np.sum(gc[es, 2] * u) + np.sum(gd[es, 2]) / nz for es, u in layout])


def _small_hybrid(rad, G):
    h, poles, _, pc = MD.hybrid_undulator(rad, n_pairs=G["n_pairs"], pole_div=tuple(G["pole_div"]),
                                          block_div=tuple(G["block_div"]))
    pts = MD.hybrid_points(n=G["n_points"], n_pairs=G["n_pairs"])
    W = np.random.default_rng(G["w_seed"]).normal(size=pts.shape)
    return h, poles, pc, pts, W


def _check_fd(G, got):
    fd = np.array([G["grad_dz"][str(k)][-1] for k in range(G["n_pairs"])])
    scale = np.abs(fd).max()
    assert np.abs(got - fd).max() <= 5e-4 * scale, (got, fd)


def test_reference_differences_have_settled():
    G = _golden()
    for k, (a, b) in G["grad_dz"].items():
        assert abs(a - b) <= 2e-4 * max(abs(v[-1]) for v in G["grad_dz"].values()), k


def test_oracle_pole_thickness_gradient_matches_reference_differences(rad):
    G = _golden()
    h, poles, pc, pts, W = _small_hybrid(rad, G)
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    N = O.assemble(pack)
    M = AO.solve_newton(pack, N, O.extfield(pack))
    L = float(np.sum(AO.field_of(pack, M, pts, 0) * W))
    assert abs(L - G["loss"]) <= 1e-5 * abs(G["loss"])
    g = AO.gradients(pack, M, pts, W)
    got = _chain(_pole_layout(rad, pack.leaves, poles, pc, G["pole_div"]), g["c"], g["d"], G["pole_div"][2])
    _check_fd(G, got)


@pytest.mark.gpu
def test_device_pole_thickness_gradient_matches_reference_differences(cuda, rad):
    from radiacuda_b200 import adjoint as A
    G = _golden()
    h, poles, pc, pts, W = _small_hybrid(rad, G)
    prob = A.FieldProblem(h, pts, "b")
    L = float(np.sum(prob.forward() * W))
    assert abs(L - G["loss"]) <= 1e-5 * abs(G["loss"])
    g = prob.backward(W)
    got = _chain(_pole_layout(rad, prob.pack.leaves, poles, pc, G["pole_div"]), g["centre"], g["dims"],
                 G["pole_div"][2])
    _check_fd(G, got)


@pytest.mark.gpu
def test_device_pole_thickness_gradient_full_hybrid(cuda, rad):
    """6,080 elements, 10,000 points: three poles against device central
    differences of the same forward pass (steps 1e-3 and 5e-4 mm)."""
    from radiacuda_b200 import adjoint as A
    pole_div = (4, 4, 4)
    h, poles, _, pc = MD.hybrid_undulator(rad)
    pts = MD.hybrid_points(n=10_000)
    W = np.random.default_rng(23).normal(size=pts.shape)
    prob = A.FieldProblem(h, pts, "b")
    assert prob.n == 6080
    F0 = prob.forward()
    assert prob.last_status["forward"][0] <= 1e-12
    g = prob.backward(W)
    assert prob.last_status["adjoint"][0] <= 1e-12
    layout = _pole_layout(rad, prob.pack.leaves, poles, pc, pole_div)
    got = _chain(layout, g["centre"], g["dims"], pole_div[2])
    scale = np.abs(got).max()
    assert scale > 0 and np.isfinite(F0).all()
    rng = np.random.default_rng(29)
    for k in rng.choice(len(poles), 3, replace=False):
        es, u = layout[k]
        fds = []
        for step in (1e-3, 5e-4):
            vals = []
            for s in (1.0, -1.0):
                c = prob.centre0.copy()
                d = prob.dims0.copy()
                c[es, 2] += s * step * u
                d[es, 2] += s * step / pole_div[2]
                vals.append(float(np.sum(prob.forward(centre=c, dims=d) * W)))
            fds.append((vals[0] - vals[1]) / (2 * step))
        assert abs(fds[0] - fds[1]) <= 1e-6 * scale, (k, fds)
        assert abs(got[k] - fds[1]) <= 1e-5 * scale, (k, got[k], fds)


@pytest.mark.gpu
def test_autograd_full_undulator_12_of_480_parameters(cuda, rad):
    import torch

    from radiacuda_b200 import adjoint as A

    h, blocks = MD.undulator(rad)
    pts = MD.undulator_points()
    prob = A.FieldProblem(h, pts, "b")
    assert prob.n == 640 and len(blocks) == 80
    ksi = prob.linear_ksi()
    blk_of = np.zeros(prob.n, dtype=np.int64)
    for b, hb in enumerate(blocks):
        blk_of[prob.elements_of(hb)] = b
    nb = len(blocks)
    mr_blk0 = np.array([prob.mr0[blk_of == b][0] for b in range(nb)])
    z = torch.tensor(pts[:, 2])
    target = 0.8 * torch.sin(2 * np.pi * z / 20.0)
    bo = torch.as_tensor(blk_of)

    def loss_of(mr_blk, dc_blk):
        mr = mr_blk[bo]
        chi = A.FieldProblem.aniso_chi(mr, ksi)
        centre = torch.as_tensor(prob.centre0) + dc_blk[bo]
        B = A.relaxed_field(prob, mr, chi, centre, torch.as_tensor(prob.dims0))
        return torch.sum((B[:, 1] - target) ** 2)

    mr_blk = torch.tensor(mr_blk0, requires_grad=True)
    dc_blk = torch.zeros((nb, 3), dtype=torch.float64, requires_grad=True)
    loss_of(mr_blk, dc_blk).backward()
    assert prob.last_status["adjoint"][0] <= 1e-12
    rng = np.random.default_rng(41)
    picks = rng.choice(nb * 6, 12, replace=False)
    for p in picks:
        b, r = divmod(int(p), 6)
        which, a = ("mr", r) if r < 3 else ("dc", r - 3)
        vals = []
        for s in (1, -1):
            m = torch.tensor(mr_blk0)
            d = torch.zeros((nb, 3), dtype=torch.float64)
            (m if which == "mr" else d)[b, a] += s * 1e-6
            with torch.no_grad():
                vals.append(float(loss_of(m, d)))
        fd = (vals[0] - vals[1]) / 2e-6
        grad = mr_blk.grad if which == "mr" else dc_blk.grad
        assert abs(float(grad[b, a]) - fd) <= 1e-5 * float(grad.abs().max()), (which, b, a, float(grad[b, a]), fd)
