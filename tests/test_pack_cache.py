"""The packed-source cache returns exactly what a fresh packing returns:
after a magnetization change, after added transformations and container
members, and with returned arrays that callers may modify."""
import numpy as np

import models as MD
from radiacuda_b200 import model


def _fresh(rad, h):
    model.clear_source_cache()
    return model.pack_sources(rad._objs, h, tuple(rad._rand))


def _same(a, b):
    return sorted(a) == sorted(b) and all(a[k].shape == b[k].shape and np.array_equal(a[k], b[k]) for k in a)


def test_cache_follows_magnetization_transforms_and_members(rad):
    h = MD.mixed_sym(rad)
    g0 = model.pack_sources(rad._objs, h, tuple(rad._rand))
    g0["poly"][:] = -7.0                         # callers may modify what they get
    assert _same(model.pack_sources(rad._objs, h, tuple(rad._rand)), _fresh(rad, h))
    leaves = model.collect_leaves(rad._objs, h)
    for k, lf in enumerate(leaves):
        if hasattr(lf.obj, "m"):
            lf.obj.m = np.array([0.1 * k, -0.2, 0.3])
    assert _same(model.pack_sources(rad._objs, h, tuple(rad._rand)), _fresh(rad, h))
    rad.TrfOrnt(h, rad.TrfRot([1, 2, 3], [0, 1, 1], 0.4))
    assert _same(model.pack_sources(rad._objs, h, tuple(rad._rand)), _fresh(rad, h))
    extra = rad.ObjRecMag([90, 0, 0], [2, 2, 2], [0, 0, 1])
    rad.ObjAddToCnt(h, [extra])
    assert _same(model.pack_sources(rad._objs, h, tuple(rad._rand)), _fresh(rad, h))
    rad.FldLenRndSw("on")
    try:
        assert _same(model.pack_sources(rad._objs, h, tuple(rad._rand)), _fresh(rad, h))
    finally:
        rad.FldLenRndSw("off")


def _same_pack(a, b):
    return (_same(a.elems, b.elems) and ((a.ext is None and b.ext is None) or _same(a.ext, b.ext))
            and all(np.array_equal(getattr(a, k), getattr(b, k)) for k in ("elem_src", "mat_kind", "mat", "mh"))
            and [id(lf.obj) for lf in a.leaves] == [id(lf.obj) for lf in b.leaves])


def test_interaction_cache_follows_magnetization_and_materials(rad):
    h = MD.mixed_sym(rad)
    rand = tuple(rad._rand)
    p0 = model.pack_interaction(rad._objs, h, 0, rand)
    p0.mat[:] = 0.0
    model.clear_source_cache()
    assert _same_pack(model.pack_interaction(rad._objs, h, 0, rand), model.pack_interaction(rad._objs, h, 0, rand))
    for k, lf in enumerate(model.collect_leaves(rad._objs, h)):
        if hasattr(lf.obj, "m"):
            lf.obj.m = np.array([0.2, 0.1 * k, -0.4])
    cached = model.pack_interaction(rad._objs, h, 0, rand)
    model.clear_source_cache()
    assert _same_pack(cached, model.pack_interaction(rad._objs, h, 0, rand))
    rad.MatApl(h, rad.MatLin([0.3, 0.1], [0.0, 0.0, 1.0]))
    cached = model.pack_interaction(rad._objs, h, 0, rand)
    model.clear_source_cache()
    assert _same_pack(cached, model.pack_interaction(rad._objs, h, 0, rand))


def test_interaction_cache_refreshes_magnetization_dependent_records(rad):
    """A linear material given by |Mr| takes its easy axis from each element's
    magnetization, so its records change with M on a cache hit; a material
    with a fixed Mr vector shares one record among its elements."""
    h = MD.mixed_sym(rad)
    rand = tuple(rad._rand)
    leaves = model.collect_leaves(rad._objs, h)
    half = len(leaves) // 2
    m_abs = rad.MatLin([0.3, 0.1], 1.1)               # easy axis along each element's M
    m_vec = rad.MatLin([0.05, 0.15], [0.0, 0.6, 0.8])  # fixed easy axis
    for k, lf in enumerate(leaves):
        lf.obj.m = np.array([0.3, 0.1 * (k + 1), 0.5])  # the |Mr| law needs a magnetization to take its axis from
        rad.MatApl(lf.handle, m_abs if k < half else m_vec)
    model.pack_interaction(rad._objs, h, 0, rand)
    for k, lf in enumerate(leaves):
        lf.obj.m = np.array([np.cos(0.3 * k), np.sin(0.3 * k), 0.2])
    cached = model.pack_interaction(rad._objs, h, 0, rand)
    model.clear_source_cache()
    fresh = model.pack_interaction(rad._objs, h, 0, rand)
    assert _same_pack(cached, fresh)
    assert not np.array_equal(cached.mat[0], cached.mat[1])  # the |Mr| records differ per element
