"""UtiDmp / UtiDmpPrs: object trees and the device state of an interaction
survive a dump and a restore (the reference dumps the object tree,
radintrc.cpp:1516,1946; the interaction state -- matrix, external field,
magnetization, LU factors -- is this library's addition, so that a solution
state outlives the process without reassembly)."""
import pickle

import numpy as np
import pytest

import models as MD
from radiacuda_b200 import model

import oracle.oracle as O


def _geom(rad, h):
    return model.pack_sources(rad._objs, h, tuple(rad._rand))


@pytest.mark.parametrize("builder", [MD.sym_blocks, MD.mixed_sym, MD.thckpgn_model])
def test_object_tree_round_trip(rad, builder):
    h = builder(rad)
    g0 = _geom(rad, h)
    h2 = rad.UtiDmpPrs(rad.UtiDmp(h, "bin"))
    assert h2 != h
    g1 = _geom(rad, h2)
    assert sorted(g0) == sorted(g1)
    for k in g0:
        assert np.array_equal(g0[k], g1[k]), k
    P = np.random.default_rng(4).uniform(-40, 60, size=(20, 3)) + 0.0137
    assert np.array_equal(O.field(g0, P, 0), O.field(g1, P, 0))
    assert rad.ObjM(h2) == rad.ObjM(h)
    # the copy is independent: changing it leaves the original alone
    leaf = model.collect_leaves(rad._objs, h2)[0]
    before = rad.ObjM(h)
    leaf.obj.m = leaf.obj.m + 1.0
    assert rad.ObjM(h) == before


def test_list_dump_and_text_form(rad):
    a = rad.ObjRecMag([0, 0, 0], [1, 2, 3], [0.1, 0.2, 0.3])
    b = rad.ObjBckg([0, 0, 1])
    out = rad.UtiDmpPrs(rad.UtiDmp([a, b], "bin"))
    assert isinstance(out, list) and len(out) == 2
    txt = rad.UtiDmp([a, b], "asc")
    assert f"Index: {a}" in txt and "background" in txt
    with pytest.raises(Exception):
        rad.UtiDmp(a, "xml")


def test_restore_refuses_foreign_pickles(rad):
    class Evil:
        def __reduce__(self):
            return (print, ("not allowed",))

    bad = rad._DMP_MAGIC + pickle.dumps({"roots": [1], "single": True, "objs": {1: Evil()}, "intrc": {}})
    with pytest.raises(Exception, match="not allowed"):
        rad.UtiDmpPrs(bad)
    with pytest.raises(Exception, match="not a dump"):
        rad.UtiDmpPrs(b"garbage")


@pytest.mark.gpu
def test_interaction_state_round_trip(rad, cuda):
    """Relaxed state, matrix and LU factors come back without reassembly."""
    h = MD.magnet_array(rad, nside=2, div=2)
    it = rad.RlxPre(h, 0, True, "f64")
    rad.RlxAuto(it, 1e-12, 200, 12)                 # FP64 LU direct solve: factors stay on the device
    M1 = np.array(rad._objs[it].M)
    N1 = rad._objs[it].native.matrix(np.float64)
    blob = rad.UtiDmp(it, "bin")
    it2 = rad.UtiDmpPrs(blob)
    I2 = rad._objs[it2]
    assert np.array_equal(I2.native.matrix(np.float64), N1)
    assert np.array_equal(I2.native.extfield(), rad._objs[it].native.extfield())
    assert np.array_equal(np.array(I2.M), M1)
    st = rad.RlxAuto(it2, 1e-12, 200, 12)
    assert np.allclose(np.array(I2.M), M1, rtol=0, atol=1e-13)
    # a relaxation started from the restored magnetization is already converged
    st = rad.RlxAuto(it2, 1e-10, 100, 4, "ZeroM->False")
    assert st[3] <= 2


@pytest.mark.gpu
def test_state_refused_for_other_geometry(rad, cuda):
    h = MD.magnet_array(rad, nside=2, div=2)
    it = rad.RlxPre(h)
    state = rad._objs[it].native.save()
    h2 = MD.sym_blocks(rad)
    pack = model.pack_interaction(rad._objs, h2, 0, tuple(rad._rand))
    from radiacuda_b200 import _native
    with pytest.raises(RuntimeError, match="stamp|sizes"):
        _native.NativeInteraction(pack, 0, state=state)
