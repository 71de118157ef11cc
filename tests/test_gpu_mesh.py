"""The mesh form of all-tetrahedron fields (unique edges and faces, csrc/mesh.cu)
against the CPU oracle and against the tetrahedra evaluated one by one.

Points outside and inside the tetrahedra (B adds the magnetization of the
tetrahedron holding the point), meshes under symmetry images (one group per
image transform), FP64 (precision 2, 1e-10 relative like the other FP64 field
tests) and FP32 terms (precision 1, 5e-5 for polyhedra)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import models as MD
from radiacuda_b200 import _native, model
from util import rel_err

import oracle.oracle as O

pytestmark = pytest.mark.gpu


def _points(rng, V, n_out=400, n_in=200):
    lo, hi = V.reshape(-1, 3).min(axis=0), V.reshape(-1, 3).max(axis=0)
    out = rng.uniform(lo - 15.0, hi + 15.0, size=(n_out, 3)) + 0.0137
    # inside: random barycentric points of random tetrahedra
    k = rng.integers(0, V.shape[0], n_in)
    w = rng.dirichlet([2.0, 2.0, 2.0, 2.0], n_in)
    ins = np.einsum("nk,nkc->nc", w, V[k])
    return np.vstack([out, ins])


def _mesh(rad, ncell, n_tets, seed):
    h, body = MD.tet_mesh(rad, ncell=ncell, n_tets=n_tets, chi=5.0)
    rng = np.random.default_rng(seed)
    for lf in model.collect_leaves(rad._objs, body):
        lf.obj.m = rng.normal(size=3)
    return h, np.asarray(MD.tet_mesh_vertices(ncell, n_tets))


@pytest.mark.parametrize("ncell,n_tets", [(3, 150), (5, 700)])
def test_mesh_form_matches_oracle_inside_and_outside(cuda, rad, ncell, n_tets):
    h, V = _mesh(rad, ncell, n_tets, 11)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    P = _points(np.random.default_rng(12), V)
    for what in (0, 1):
        got = _native.field(g, P, what, 2)
        exp = O.field(g, P, what)
        assert rel_err(got, exp) < 1e-10, what
    assert rel_err(_native.field(g, P, 0, 1), O.field(g, P, 0)) < 5e-5


def test_mesh_form_with_symmetry_images(cuda, rad):
    MD.reset(rad)
    V = np.asarray(MD.tet_mesh_vertices(3, 150)) + np.array([20.0, 3.0, 4.0])
    ids = [rad.ObjPolyhdr(v.tolist(), MD.TET_FACES) for v in V]
    body = rad.ObjCnt(ids)
    rad.MatApl(body, rad.MatLin([5.0, 5.0], [0, 0, 1e-12]))
    rad.TrfZerPerp(body, [0, 0, 0], [1, 0, 0])
    rad.TrfZerPara(body, [0, 0, 0], [0, 0, 1])
    rng = np.random.default_rng(13)
    for lf in model.collect_leaves(rad._objs, body):
        lf.obj.m = rng.normal(size=3)
    g = model.pack_sources(rad._objs, body, tuple(rad._rand))
    P = np.vstack([_points(rng, V), _points(rng, V * np.array([-1.0, 1.0, 1.0]))])
    # the oracle is the face-by-face form: the two exact FP64 forms differ at
    # the 1e-10 level when images multiply the cancellations
    for what in (0, 1):
        assert rel_err(_native.field(g, P, what, 2), O.field(g, P, what)) < 5e-10, what


def test_mesh_form_equals_tetrahedra_one_by_one(cuda):
    """Same sum, term for term: the mesh form and the per-tetrahedron form
    (RADB200_MESH_FORM=0, read once per process) agree to rounding."""
    code = (
        "import sys, numpy as np; sys.path[:0] = [{root!r}, {tests!r}]\n"
        "import models as MD\n"
        "from radiacuda_b200 import rad, model, _native\n"
        "h, body = MD.tet_mesh(rad, ncell=5, n_tets=700, chi=5.0)\n"
        "rng = np.random.default_rng(5)\n"
        "[setattr(lf.obj, 'm', rng.normal(size=3)) for lf in model.collect_leaves(rad._objs, body)]\n"
        "g = model.pack_sources(rad._objs, h, tuple(rad._rand))\n"
        "P = rng.uniform(-20, 30, size=(3000, 3)) + 0.011\n"
        "np.save(sys.argv[1], np.stack([_native.field(g, P, 0, 2), _native.field(g, P, 0, 1)]))\n"
    )
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = code.format(root=root, tests=os.path.join(root, "tests"))
    out = {}
    for flag in ("1", "0"):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"radb200_meshform_{os.getpid()}_{flag}.npy")
        env = dict(os.environ, RADB200_MESH_FORM=flag)
        r = subprocess.run([sys.executable, "-c", code, path], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[flag] = np.load(path)
        os.remove(path)
    assert rel_err(out["1"][0], out["0"][0]) < 2e-11
    assert rel_err(out["1"][1], out["0"][1]) < 2e-5
