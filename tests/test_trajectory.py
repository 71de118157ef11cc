"""Electron trajectories (rad.FldPtcTrj, radb200_trajectories) against the
reference's own FldPtcTrj (tests/golden/trajectory.json, made by
tests/golden/make_trajectory_golden.py), with the default fixed-step
integration and with the step-doubling control.

CPU tests pin the oracle's restatement of the integrator
(oracle/trajectory_oracle.py) on the oracle field; GPU tests run the device
kernel (one CTA per trajectory) through rad.FldPtcTrj.
"""
import json
import os

import numpy as np
import pytest

import models as MD
from radiacuda_b200 import model

import oracle.oracle as O
from oracle.trajectory_oracle import trajectory

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "trajectory.json")))
ADAPTIVE = GOLD["adaptive_prec"]


def tet_given(R, seed=77):
    h, body = MD.tet_mesh(R, ncell=3, n_tets=150, chi=5.0)
    rng = np.random.default_rng(seed)
    for t in R.ObjCntStuf(body):
        R.ObjSetM(t, rng.normal(scale=0.6, size=3).tolist())
    return h


BUILDERS = {
    "array_given": lambda R: MD.magnet_array(R, nside=2, div=2),
    "sym_given": MD.sym_blocks,
    "tet_given": tet_given,
    "dipole_relaxed": lambda R: MD.iron_dipole(R, n_target=300),
}


def _tol(name, ref):
    # given magnetizations: integrator rounding; relaxed: the relaxation's own
    # agreement with the reference (5e-5 saturating) carried along the orbit
    rel = 1e-8 if name.endswith("_given") else 5e-5
    return 1e-10 + rel * np.abs(ref).max(axis=0)


def _set_prec(rad, adaptive):
    if adaptive:
        rad.FldCmpPrc(f"PrcCoord->{ADAPTIVE[0]},PrcAngle->{ADAPTIVE[1]}")
    else:
        rad.FldCmpPrc("PrcCoord->-1,PrcAngle->-1")


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["array_given", "sym_given", "tet_given"])
def test_oracle_integrator_matches_reference(rad, name):
    h = BUILDERS[name](rad)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    fld = lambda p: O.field(g, p.reshape(1, 3), 0)[0]  # noqa: E731
    for run in GOLD["cases"][name]["runs"]:
        for mode in ("fixed", "adaptive"):
            prec = None if mode == "fixed" else [ADAPTIVE[0], ADAPTIVE[1], ADAPTIVE[0], ADAPTIVE[1]]
            T = trajectory(fld, run["E"], run["init"], run["lim"][0], run["lim"][1], run["np"], prec)
            ref = np.array(run[mode])
            assert np.all(np.abs(T - ref) <= _tol(name, ref)), (name, mode, np.abs(T - ref).max(axis=0))


def test_fldptctrj_argument_errors(rad):
    h = MD.magnet_array(rad, nside=2, div=2)
    with pytest.raises(Exception, match="initial conditions"):
        rad.FldPtcTrj(h, 1.0, [0, 0, 0], [0, 10], 5)
    with pytest.raises(Exception, match="Y range"):
        rad.FldPtcTrj(h, 1.0, [0, 0, 0, 0], [0, 10, 20], 5)
    with pytest.raises(Exception):
        rad.FldPtcTrj(h, -1.0, [0, 0, 0, 0], [0, 10], 5)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(BUILDERS))
@pytest.mark.parametrize("mode", ["fixed", "adaptive"])
def test_fldptctrj_matches_reference(rad, cuda, name, mode):
    h = BUILDERS[name](rad)
    solve = GOLD["cases"][name]["solve"]
    if solve is not None:
        rad.Solve(h, solve[0], solve[1], 4)
    try:
        _set_prec(rad, mode == "adaptive")
        for run in GOLD["cases"][name]["runs"]:
            T = np.array(rad.FldPtcTrj(h, run["E"], run["init"], run["lim"], run["np"]))
            ref = np.array(run[mode])
            assert T.shape == ref.shape
            assert np.all(np.abs(T - ref) <= _tol(name, ref)), (name, mode, np.abs(T - ref).max(axis=0))
    finally:
        _set_prec(rad, False)


@pytest.mark.gpu
def test_batched_trajectories_equal_single_ones(rad, cuda):
    """An [n, 4] batch runs n CTAs; each row equals the single-trajectory call."""
    h = BUILDERS["array_given"](rad)
    rng = np.random.default_rng(5)
    init = np.column_stack([rng.uniform(-20, 0, 24), rng.normal(0, 1e-3, 24), rng.uniform(6.5, 9.5, 24),
                            rng.normal(0, 1e-3, 24)])
    B = rad.FldPtcTrj(h, 0.05, init, [-60.37, 60.21], 41)
    assert B.shape == (24, 41, 5)
    for k in (0, 7, 23):
        S = np.array(rad.FldPtcTrj(h, 0.05, init[k].tolist(), [-60.37, 60.21], 41))
        assert np.array_equal(B[k], S)


@pytest.mark.gpu
def test_single_point_and_step_failure(rad, cuda):
    h = BUILDERS["array_given"](rad)
    one = rad.FldPtcTrj(h, 0.05, [-10.3, 0.001, 8.1, -0.002], [-60.37, 60.21], 1)
    assert one == [-60.37, -10.3, 0.001, 8.1, -0.002]
    # accuracy far below what doubles can hold: the step control gives up
    # (step too small or the evaluation budget), reported as the reference's error
    try:
        rad.FldCmpPrc("PrcCoord->1e-30,PrcAngle->1e-30")
        with pytest.raises(Exception, match="Radia::Error20"):
            rad.FldPtcTrj(h, 0.05, [-10.3, 0.001, 8.1, -0.002], [-60.37, 60.21], 3)
    finally:
        _set_prec(rad, False)
