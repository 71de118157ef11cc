"""radiacuda_b200 -- B200-native (sm_100a) relaxation hot path for Radia.

    from radiacuda_b200 import rad
    rad.FldLenRndSw('off')
    m = rad.ObjRecMag([0, 0, 0], [1, 1, 1], [-0.5, 1, 0.7])
    rad.Fld(m, 'b', [0.52, 0.6, 0.7])

``rad`` mirrors the reference's ``radia`` module for the hot path (object
construction, symmetries, materials, RlxPre / RlxAuto / Solve / Fld); all
numerics run in libradb200 (include/radb200.h) on the GPU.
"""
from . import rad  # noqa: F401

__all__ = ["rad"]
