"""Generates tests/golden/baseline_configs.npz: reference Radia fields on the
five benchmark configurations, at their stated sizes.

    make -f oracle/Makefile.ref -j8                # builds oracle/_ref
    python tests/golden/make_baseline_golden.py [c1 c2 c3 c3o c3q c4 c5]

Runs the reference Radia CPU module (oracle/_ref, FldLenRndSw('off')) on the
seeded models of tests/models.py:

  c1  432 anisotropic blocks, Solve(prec 1e-10, method 4), B at the 10,000
      grid points 5 mm above the array;
  c2  the 4,000-block saturating dipole (2 mirror planes, racetrack),
      Solve(prec 1e-7, method 4: the reference's FP32 matrix puts the floor
      of its misfit near there), B at a seeded 10,000-point subsample of the
      100^3 gap grid;
  c3  a 3,000-tetrahedron mesh of the 20k model's construction at chi = 1000:
      the FP64 interaction matrix built column by column from the reference's
      own field of each element magnetized by a unit vector (Fld 'h' at the
      element centres), solved in FP64 (LAPACK), and B of that solution at
      2,000 points outside the body -- the FP64 oracle of the direct-solve
      path (the reference stores its own matrix in FP32, which is not a 1e-6
      oracle at chi = 1000);
  c3o the same 3,000-tetrahedron system built and solved by the CPU oracle
      (oracle/oracle.py: the interaction matrix of the restated element
      fields, LAPACK, B by the oracle field) -- the FP64 oracle proper;
  c3q the reference's self-interaction block of each of those tetrahedra,
      kept for the elements where it departs from the oracle's by more than
      1e-9 (one element, whose nearly axis-parallel edge sends the reference
      into a tolerance branch; tests/test_oracle_quadrature.py settles which
      of the two is right with an independent surface-charge quadrature);
  c4  the 640-block planar undulator, Solve(prec 1e-10), B at 4,000 axis points;
  c5  the 6,080-element hybrid undulator (saturating poles, a mirror plane),
      Solve(prec 1e-7), B at a seeded 10,000-point subsample of its 1e5 points.

Field evaluations and the matrix columns of c3 are split over worker
processes forked after the model is built and solved.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)

import models as MD  # noqa: E402
import radia as R  # noqa: E402

OUT = os.path.join(HERE, "baseline_configs.npz")
NPROC = min(8, os.cpu_count() or 1)
_MODEL = [0]


def _fld_slice(args):
    what, P = args
    return np.array(R.Fld(_MODEL[0], what, P.tolist())).reshape(-1, 3)


def field_parallel(model, what, P):
    _MODEL[0] = model
    parts = np.array_split(P, NPROC * 4)
    with mp.get_context("fork").Pool(NPROC) as pool:
        res = pool.map(_fld_slice, [(what, p) for p in parts if len(p)])
    return np.concatenate(res, axis=0)


def subsample(P, n, seed):
    idx = np.sort(np.random.default_rng(seed).choice(P.shape[0], n, replace=False))
    return idx, P[idx]


def solve(model, prec, iters):
    t = time.time()
    st = R.Solve(model, prec, iters, 4)
    print(f"  solve {time.time() - t:.1f} s, misfit {st[0]:.3e}, iterations {st[3]:.0f}")
    return np.array(st)


def c1(out):
    m = MD.magnet_array(R)
    P = MD.magnet_array_points()
    out["c1_status"] = solve(m, 1e-10, 10000)
    out["c1_b"] = field_parallel(m, "b", P)


def c2(out):
    m = MD.iron_dipole(R, n_target=4000)
    idx, P = subsample(MD.iron_dipole_points(100), 10000, 22)
    out["c2_status"] = solve(m, 1e-7, 6000)
    out["c2_idx"] = idx
    out["c2_b"] = field_parallel(m, "b", P)


# --- c3: the FP64 interaction matrix from the reference's own element fields
_C3 = {}


def _columns(js):
    elems, cen = _C3["elems"], _C3["cen"]
    cols = np.zeros((len(js), 3, cen.shape[0], 3))
    for a, j in enumerate(js):
        for k in range(3):
            e = [0.0, 0.0, 0.0]
            e[k] = 1.0
            R.ObjSetM(elems[j], e)
            cols[a, k] = np.array(R.Fld(elems[j], "h", cen.tolist())).reshape(-1, 3)
        R.ObjSetM(elems[j], [0.0, 0.0, 0.0])
    return js, cols


def c3(out, n_tets=3000, ncell=8, chi=1000.0, n_pts=2000):
    whole, body = MD.tet_mesh(R, ncell=ncell, n_tets=n_tets, chi=chi)
    V = np.asarray(MD.tet_mesh_vertices(ncell, n_tets))
    elems = R.ObjCntStuf(body)
    assert len(elems) == n_tets
    cen = V.mean(axis=1)
    n = n_tets
    for e in elems:
        R.ObjSetM(e, [0.0, 0.0, 0.0])
    _C3.update(elems=elems, cen=cen)
    t = time.time()
    N = np.zeros((3 * n, 3 * n))
    chunks = np.array_split(np.arange(n), NPROC * 8)
    with mp.get_context("fork").Pool(NPROC) as pool:
        for js, cols in pool.imap_unordered(_columns, chunks):
            for a, j in enumerate(js):
                for k in range(3):
                    N[:, 3 * j + k] = cols[a, k].reshape(-1)
    print(f"  c3 matrix {time.time() - t:.1f} s")
    mr = np.tile([0.0, 0.0, 1e-12], n)
    hext = np.tile([0.0, 0.0, 1.0], n)  # the 1 T background (H = B outside material)
    A = np.eye(3 * n) - chi * N
    t = time.time()
    M = np.linalg.solve(A, chi * hext + mr)
    res = np.abs(A @ M - (chi * hext + mr)).max() / np.abs(chi * hext + mr).max()
    print(f"  c3 solve {time.time() - t:.1f} s, relative residual {res:.2e}")
    for i, e in enumerate(elems):
        R.ObjSetM(e, M[3 * i:3 * i + 3].tolist())
    P = MD.tet_mesh_points(n_pts, ncell=ncell)
    out["c3_M"] = M
    out["c3_b"] = field_parallel(whole, "b", P)
    out["c3_residual"] = np.array([res])


def _oracle_c3_pack(n_tets=3000, ncell=8, chi=1000.0):
    from oracle import oracle as O
    from radiacuda_b200 import model, rad
    whole, body = MD.tet_mesh(rad, ncell=ncell, n_tets=n_tets, chi=chi)
    return O, model, rad, whole, model.pack_interaction(rad._objs, whole, 0, tuple(rad._rand))


def c3o(out, n_pts=2000, ncell=8):
    O, model, rad, whole, pack = _oracle_c3_pack(ncell=ncell)
    N = O.assemble(pack)
    M = O.linear_direct(pack, N, O.extfield(pack))
    for lf, m in zip(pack.leaves, M.reshape(-1, 3)):
        lf.obj.m = m.copy()
    P = MD.tet_mesh_points(n_pts, ncell=ncell)
    out["c3o_M"] = M
    out["c3o_b"] = O.field(model.pack_sources(rad._objs, whole, tuple(rad._rand)), P, 0)


def c3q(out, ncell=8, n_tets=3000):
    O, _, _, _, pack = _oracle_c3_pack(ncell=ncell, n_tets=n_tets)
    N = O.assemble(pack)
    _, body = MD.tet_mesh(R, ncell=ncell, n_tets=n_tets, chi=1000.0)
    V = np.asarray(MD.tet_mesh_vertices(ncell, n_tets))
    elems = R.ObjCntStuf(body)
    cen = V.mean(axis=1)
    for e in elems:
        R.ObjSetM(e, [0.0, 0.0, 0.0])
    idx, blocks = [], []
    for j, e in enumerate(elems):
        blk = np.zeros((3, 3))
        for k in range(3):
            m = [0.0, 0.0, 0.0]
            m[k] = 1.0
            R.ObjSetM(e, m)
            blk[:, k] = R.Fld(e, "h", cen[j].tolist())
        R.ObjSetM(e, [0.0, 0.0, 0.0])
        if np.abs(blk - N[3 * j:3 * j + 3, 3 * j:3 * j + 3]).max() > 1e-9:
            idx.append(j)
            blocks.append(blk)
    out["c3q_idx"] = np.array(idx, dtype=np.int64)
    out["c3q_ref"] = np.array(blocks).reshape(-1, 3, 3)
    out["c3q_V"] = V[idx].reshape(-1, 4, 3)
    print(f"  reference self blocks off the oracle's by > 1e-9: elements {idx}")


def c4(out):
    m, _ = MD.undulator(R)
    P = MD.undulator_points()
    out["c4_status"] = solve(m, 1e-10, 10000)
    out["c4_b"] = field_parallel(m, "b", P)


def c5(out):
    m = MD.hybrid_undulator(R)[0]
    idx, P = subsample(MD.hybrid_points(), 10000, 55)
    out["c5_status"] = solve(m, 1e-7, 6000)
    out["c5_idx"] = idx
    out["c5_b"] = field_parallel(m, "b", P)


def main(names):
    out = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    for nm in names:
        t = time.time()
        print(nm, flush=True)
        globals()[nm](out)
        print(f"  {nm} done in {time.time() - t:.1f} s", flush=True)
        np.savez_compressed(OUT, **out)
        print("wrote", OUT, flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["c1", "c2", "c3", "c3o", "c3q", "c4", "c5"])
