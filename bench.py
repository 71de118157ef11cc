"""Benchmark of the relaxation hot path on the 20k-tetrahedron model.

Workload (one step): the precision model -- 20,000 tetrahedra from a seeded
jittered Kuhn lattice with 2% slivers, linear isotropic chi = 1000 in a
uniform 1 T background field, a dense 60,000 x 60,000 interaction system --
assembled on the device, solved by the mixed-precision direct solver (TF32
tensor-core LU + FP64 GMRES refinement), then B evaluated at 1,000,000
points outside the body.  Metric: seconds per solve+Fld step (lower is
better), with the B error of the step against the plain FP64 GPU path
(FP64 assembly, FP64 LU, FP64 field) reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: the path does not shard without a per-matvec exchange, so N GPUs
run N independent replicas (weak scaling); the step time is the max over
ranks.  Timing: CUDA events on the default stream (the library's stream),
L2 flushed before every step, clocks sampled during the timed region.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "solve+Fld time at <=1e-6 rel B err vs plain FP64 GPU; adjoint/forward time ratio"
WORKLOAD = dict(workload="tet20k: 20,000 tetrahedra (2% slivers), linear chi=1000, 1 T background, "
                         "dense 60,000^2 system, B at 1e6 points outside the body",
                n_tets=20000, n_points=1_000_000, chi=1000.0)
NCELL = 15
MIXED_FAST = 2 | 16   # RADB200_STORE_MIXED | RADB200_ASM_FAST
F64_FAST = 1 | 16     # RADB200_STORE_F64 | RADB200_ASM_FAST
# field of the mixed step: vertex/edge tetrahedron form with FP32 terms, FP64
# vertex offsets and FP64 accumulation (radb200_field precision 1); its B
# error against the plain FP64 path is reported with every run
FIELD_PREC = 1
# plain FP64 comparator: the fastest exact FP64 kernels -- vertex/edge
# assembly stored in FP64, FP64 LU, vertex/edge field in FP64 (precision 2)
PLAIN_FIELD_PREC = 2
PLAIN_REPS = 3


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, out):
        self.out = out
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.out, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
            # the sampler's start-up (driver initialisation) stalls the GPU for
            # a moment: time nothing until its first sample is written
            t0 = time.time()
            while time.time() - t0 < 5.0 and self.p.poll() is None:
                self.f.flush()
                if os.path.getsize(self.out) > 0:
                    break
                time.sleep(0.05)
            time.sleep(0.5)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self, dev=0):
        try:
            rows = [r.split(",") for r in open(self.out).read().strip().splitlines()]
            rows = [[x.strip() for x in r] for r in rows if r and r[0].strip() == str(dev)]
            sm = [float(r[1]) for r in rows]
            mx = float(rows[0][2]) if rows else None
            reasons = set()
            for r in rows:
                for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                    "samples": len(sm)}
        except Exception as e:  # pragma: no cover
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "error": str(e)}


def max_over_ranks(value, device):
    """The job's step time under N replicas: the slowest rank's device time
    (all-reduce MAX over the default process group; NCCL on GPUs, gloo on CPU)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def b_errors(got, exp):
    """(max-norm ratio, largest per-point ratio) of B against a reference
    field; per point |dB_i| / |B_i|, points with |B_i| below 1e-3 of the
    largest measured against that floor."""
    g = np.asarray(got, dtype=float).reshape(-1, 3)
    e = np.asarray(exp, dtype=float).reshape(-1, 3)
    n = np.linalg.norm(e, axis=1)
    d = np.linalg.norm(g - e, axis=1)
    return float(np.abs(g - e).max() / np.abs(e).max()), float((d / np.maximum(n, 1e-3 * n.max())).max())


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, rank, world):
    import torch
    from radiacuda_b200 import _abi, _native, model, rad
    import models as MD

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    L = _native.lib()
    L.radb200_measure_fma_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    fp64_peak, fp32_peak = C.c_double(0), C.c_double(0)
    _native.check(L.radb200_measure_fma_peak(1, C.byref(fp64_peak)), "fma peak")
    _native.check(L.radb200_measure_fma_peak(0, C.byref(fp32_peak)), "fma peak")

    m, body = MD.tet_mesh(rad, ncell=NCELL, n_tets=WORKLOAD["n_tets"], chi=WORKLOAD["chi"])
    P = MD.tet_mesh_points(WORKLOAD["n_points"], ncell=NCELL)
    pack = model.pack_interaction(rad._objs, m, 0, tuple(rad._rand))
    src = model.pack_sources(rad._objs, m, tuple(rad._rand))
    # element e -> polyhedron row of the field geometry (same traversal order)
    poly_rows = np.arange(pack.elem_src.shape[0])
    n3 = 3 * pack.elem_src.shape[0]
    gE = _abi.GeomHolder(pack.elems)
    gR = _abi.RelaxHolder(pack.elem_src, pack.mat_kind, pack.mat, pack.mh)
    gX = _abi.GeomHolder(pack.ext)
    d_pts = torch.from_numpy(P).to(dev)
    d_B = torch.empty_like(d_pts)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    Mbuf = np.zeros(n3)
    st = np.zeros(4)
    _dp = C.POINTER(C.c_double)

    def step(mode, storage, fprec, ev=None):
        h = C.c_int64(0)
        if ev:
            ev[0].record()
        _native.check(L.radb200_intrc_create(C.cast(gE.ptr, C.c_void_p), C.cast(gR.ptr, C.c_void_p),
                                             C.cast(gX.ptr, C.c_void_p), storage, C.byref(h)), "intrc_create")
        if ev:
            ev[1].record()
        _native.check(L.radb200_direct_solve(h.value, mode, 1e-12 if mode == 0 else 1e-13, 200,
                                             Mbuf.ctypes.data_as(_dp), st.ctypes.data_as(_dp)), "direct_solve")
        L.radb200_intrc_free(h.value)
        src["poly"][poly_rows, 3:6] = Mbuf.reshape(-1, 3)
        if ev:
            ev[2].record()
        _native.field_dev(src, d_pts.data_ptr(), P.shape[0], 0, d_B.data_ptr(), fprec)
        if ev:
            ev[3].record()
        return st.copy()

    # plain FP64 GPU path: the error reference and the speed comparator, one
    # warm-up then PLAIN_REPS steps timed with CUDA events like the mixed step
    # (--no-plain skips it, for launch-list captures of the mixed step alone)
    t_plain, B_plain, plain_phases, plain_reps = float("nan"), None, {}, []
    if not args.no_plain:
        step(0, F64_FAST, PLAIN_FIELD_PREC)
        pa, ps, pf = [], [], []
        for _ in range(PLAIN_REPS):
            flush.fill_(3.0)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            step(0, F64_FAST, PLAIN_FIELD_PREC, ev)
            torch.cuda.synchronize()
            pa.append(ev[0].elapsed_time(ev[1]) / 1e3)
            ps.append(ev[1].elapsed_time(ev[2]) / 1e3)
            pf.append(ev[2].elapsed_time(ev[3]) / 1e3)
            plain_reps.append(ev[0].elapsed_time(ev[3]) / 1e3)
        t_plain = float(np.median(plain_reps))
        plain_phases = {"assembly": round(float(np.median(pa)), 4), "solve": round(float(np.median(ps)), 4),
                        "field": round(float(np.median(pf)), 4)}
        B_plain = d_B.cpu().numpy().copy()

    launches0 = _native.kernel_launches()
    for _ in range(args.warmup):
        flush.fill_(1.0)
        step(1, MIXED_FAST, FIELD_PREC)
    torch.cuda.synchronize()
    B_mixed = d_B.cpu().numpy().copy()
    err, err_pp = b_errors(B_mixed, B_plain) if B_plain is not None else (None, None)

    times, t_asm, t_solve, t_fld = [], [], [], []
    # the raw samples go to BENCH_CLOCKS_DIR (default: the temp directory); the
    # JSON line carries their summary
    clocks = Clocks(os.path.join(os.environ.get("BENCH_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"bench_clocks_r{rank}.csv"))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    launches_before = _native.kernel_launches()
    L.radb200_update_stats.argtypes = [C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double)]
    L.radb200_update_timing(1)
    with clocks:
        for _ in range(args.steps):
            flush.fill_(2.0)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            step(1, MIXED_FAST, FIELD_PREC, ev)
            torch.cuda.synchronize()
            t_asm.append(ev[0].elapsed_time(ev[1]) / 1e3)
            t_solve.append(ev[1].elapsed_time(ev[2]) / 1e3)
            t_fld.append(ev[2].elapsed_time(ev[3]) / 1e3)
            times.append(ev[0].elapsed_time(ev[3]) / 1e3)
    launches = (_native.kernel_launches() - launches_before) // max(args.steps, 1)
    upd_n, upd_s, upd_b, upd_f = C.c_int64(0), C.c_double(0), C.c_double(0), C.c_double(0)
    L.radb200_update_stats(C.byref(upd_n), C.byref(upd_s), C.byref(upd_b), C.byref(upd_f))
    L.radb200_update_timing(0)
    torch.cuda.synchronize()
    t_step = float(np.mean(times))
    if world > 1:
        t_step = max_over_ranks(t_step, dev)

    # end to end through the public API with host buffers (rad.RlxPre/RlxAuto/Fld)
    Ph = torch.from_numpy(P).pin_memory().numpy()
    e2e = []
    for _ in range(0 if args.profile else max(1, min(args.steps, 2))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        im = rad.RlxPre(m, storage="mixed", fast=True)
        rad.RlxAuto(im, 1e-13, 200, 13)
        Bh = rad.Fld(m, "b", Ph, precision="single")
        torch.cuda.synchronize()
        e2e.append(time.perf_counter() - t0)
        rad.UtiDel(im)
    e2e_err = b_errors(Bh, B_plain) if (e2e and B_plain is not None) else None
    if not e2e:
        e2e = [float("nan")]

    # roofline of the LU trailing update (tcgen05 GEMM, K = the panel width): its flops
    # (2 m^2 K per launch) over the event-timed launch durations, against the
    # dense rate of its operand type (FP16: the measured bf16 rate; TF32: half
    # of it); the HBM side (C read + written, panels once) beside it
    peaks = _peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    # the trailing update runs inside a seconds-long step: the sustained rate
    # (a GEMM loop under the power cap) is its denominator
    bf16 = peaks.get("bf16_tflops_sustained")
    # which GEMM the LU ran: 3 = TMA-fed with scaled FP16 operands (the dense
    # FP16 rate equals the bf16 one), 2 = TMA-fed with TF32 operands (half of it)
    L.radb200_tc_selftest.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double)]
    tc_state, tc_err = C.c_int(0), C.c_double(0.0)
    L.radb200_tc_selftest(C.byref(tc_state), C.byref(tc_err))
    f16_ops = tc_state.value == 3
    div = 1.0 if f16_ops else 2.0
    tf32_peak = float(bf16) / div if bf16 else 1400.0 / div
    upd_tflops = upd_f.value / max(upd_s.value, 1e-30) / 1e12
    upd_gbs = upd_b.value / max(upd_s.value, 1e-30) / 1e9
    upd_bytes_per_launch = upd_b.value / max(upd_n.value, 1)
    roof_upd = {"kernel": ("tc_update_tma_kernel<FP16 operands> (LU trailing update A22 -= L21 U12, K = 1024, "
                           "then 768 for the last 30,000 rows; operands scaled per row and column by powers of two, "
                           "FP32 accumulation)" if f16_ops else
                           "tc_update_tma_kernel<TF32 operands> (LU trailing update A22 -= L21 U12, K = 1024, "
                           "then 768 for the last 30,000 rows)"),
                "bound": "tensor",
                "achieved": round(upd_tflops, 1), "peak": round(tf32_peak, 1), "unit": "TFLOP/s",
                "frac": round(upd_tflops / tf32_peak, 4),
                "peak_source": (("measured sustained bf16 dense (the FP16 rate)" if f16_ops else
                                 "measured sustained bf16 dense / 2 (TF32 runs at half the bf16 rate)") if bf16 else
                                "fallback sustained bf16" + ("" if f16_ops else " / 2")),
                "frac_of_burst": round(upd_tflops / (float(peaks.get("bf16_tflops", 1590.0)) / div), 4),
                "hbm_achieved_gbs": round(upd_gbs, 1), "hbm_peak_gbs": hbm, "hbm_frac": round(upd_gbs / hbm, 4),
                "traffic": round(TC_TRAFFIC_OVER_ALGORITHMIC["f16" if f16_ops else "tf32"] * upd_bytes_per_launch),
                "traffic_note": "ncu dram bytes / algorithmic bytes (0.92) of the same kernel on a 9,000^2 LU, "
                                "times the algorithmic bytes per launch",
                "launches_per_step": int(upd_n.value // max(args.steps, 1)),
                "seconds_per_step": round(upd_s.value / max(args.steps, 1), 4),
                "algorithmic": ("2 m^2 K flops; 8 m^2 + 4 m K bytes per launch (FP32 C read + written, FP16 panels "
                                "read once)" if f16_ops else
                                "2 m^2 K flops; 8 m^2 + 8 m K bytes per launch (FP32 C read + written, panels read once)")}
    # the field kernel (FP64 pipe, transcendental-bound) against the measured FP64 FMA peak
    n_tets = src["poly"].shape[0]
    fld_s = float(np.mean(t_fld))
    achieved = P.shape[0] * n_tets * FIELD_OPS_PER_TET / fld_s / 1e12
    clk = clocks.summary(int(os.environ.get("LOCAL_RANK", 0)))
    res = {
        "metric": METRIC, "value": round(t_step, 4), "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t_step, 2), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f16+f32" if f16_ops else "f64+tf32+f32", "data": "synthetic (seeded)",
        "config": dict(WORKLOAD, parallelism=f"replicas{world}", l2="flushed (256 MB write) before every step",
                       solver=("LU with FP32 factors, tensor-core updates on scaled FP16 operands (FP32 accumulation), FP64 GMRES-IR"
                               if f16_ops else "TF32 LU + FP64 GMRES-IR"), field="vertex/edge tetrahedron form, FP32 terms, FP64 vertex offsets and accumulation",
                       assembly="FP64 vertex/edge form, stored FP32 with the FP64 residue of near blocks"),
        "breakdown_s": {"assembly": round(float(np.mean(t_asm)), 4), "solve": round(float(np.mean(t_solve)), 4),
                        "field": round(fld_s, 4)},
        "steps_s": {"total": [round(x, 4) for x in times], "assembly": [round(x, 4) for x in t_asm],
                    "solve": [round(x, 4) for x in t_solve], "field": [round(x, 4) for x in t_fld]},
        "b_rel_err_vs_plain_fp64": err, "b_rel_err_per_point_vs_plain_fp64": err_pp,
        "b_err_note": ("max|dB| / max|B| and max_i |dB_i| / |B_i| over the 1e6 points against the plain FP64 GPU "
                       "path, which the tests pin to an FP64 oracle built from the reference's own element fields "
                       "(3,000 tetrahedra, chi = 1000, 1e-6 per point)"),
        "plain_fp64_s": round(t_plain, 4), "plain_fp64_breakdown_s": plain_phases,
        "plain_fp64_reps_s": [round(x, 4) for x in plain_reps],
        "plain_fp64_config": "FP64 vertex/edge assembly stored FP64, FP64 LU (+ FP64 refinement), FP64 vertex/edge field; "
                             "warm, CUDA-event timed, median of 3",
        "speedup_vs_plain_fp64": round(t_plain / t_step, 3),
        "e2e": {"value": round(float(np.mean(e2e)), 4), "unit": "s", "b_rel_err_vs_plain_fp64": e2e_err,
                "h2d_bytes_per_step": int(P.nbytes + sum(a.nbytes for a in src.values()) + sum(a.nbytes for a in pack.elems.values())),
                "d2h_bytes_per_step": int(P.nbytes + n3 * 8)},
        "gpu_launches": int(launches),
        "roofline": roof_upd,
        "roofline_field": field_roofline(P.shape[0] * n_tets / fld_s, achieved, fp32_peak.value, clk),
        "clocks": clk,
    }
    return res


def adjoint_ratio(reps=5):
    """Second half of the metric: wall time of one full adjoint gradient over
    one forward solve, through radiacuda_b200.adjoint.FieldProblem (the public
    API: host parameters in, host field / gradients out), on
      planar undulator: 2 x 40 blocks 50x10x5 mm, anisotropic MatLin, 2x2x2
        subdivision (640 elements), B at 4,000 on-axis points, FP64 direct solve;
      hybrid undulator: 80 NdFeB blocks + 80 saturating iron poles (4x4x4),
        about 6,000 elements, mirror plane (2 images), B at 1e5 points,
        Newton-Krylov relaxation.
    Forward = assembly + solve + field; adjoint = field VJP + transposed solve
    + derivative contractions.  Median of `reps` after one warm-up; every
    rep's times and the SM clocks sampled over each case are kept, since a
    single slow rep on a shared host moves a median of few."""
    import torch

    from radiacuda_b200 import adjoint as A
    from radiacuda_b200 import rad
    import models as MD

    out = {}
    cases = [("undulator_640", lambda: MD.undulator(rad, nper_row=40, div=2)[0], MD.undulator_points(4000, 40)),
             ("hybrid_6k", lambda: MD.hybrid_undulator(rad)[0], MD.hybrid_points(100_000))]
    for name, build, pts in cases:
        h = build()
        prob = A.FieldProblem(h, pts, "b", prec=1e-12)
        W = np.random.default_rng(1).normal(size=pts.shape)
        tf, tb = [], []
        clk = Clocks(os.path.join(os.environ.get("BENCH_CLOCKS_DIR", tempfile.gettempdir()),
                                  f"radb200_adjoint_clocks_{os.getpid()}_{name}.csv"))
        with clk:
            for r in range(reps + 1):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                prob.forward()
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                prob.backward(W)
                torch.cuda.synchronize()
                t2 = time.perf_counter()
                if r:
                    tf.append(t1 - t0)
                    tb.append(t2 - t1)
        f, b = float(np.median(tf)), float(np.median(tb))
        out[name] = {"n_elements": int(prob.n), "n_points": int(pts.shape[0]), "forward_s": round(f, 4),
                     "adjoint_s": round(b, 4), "adjoint_over_forward": round(b / f, 3),
                     "forward_reps_s": [round(x, 4) for x in tf], "adjoint_reps_s": [round(x, 4) for x in tb],
                     "clocks": clk.summary(int(os.environ.get("LOCAL_RANK", 0))),
                     "phases_s": {k: round(v, 4) for k, v in prob.last_timing.items()},
                     "adjoint_residual": float(prob.last_status["adjoint"][0]),
                     "adjoint_iterations": int(prob.last_status["adjoint"][1])}
    return out


def c1_anchor(reps=3):
    """The 432-block anisotropic magnet array (16 blocks 10 mm, MatLin
    chi_par 0.06 / chi_perp 0.17, 3x3x3 subdivision) end to end through the
    public API: Solve(prec 1e-10, method 4) then B at the 10,000 grid points
    5 mm above the array.  Ours (rad.Solve + rad.Fld, host buffers) and the
    reference CPU module's same calls, both measured (median of `reps` after
    one warm-up; the reference's Fld is its serial per-point loop, 1 core),
    and the per-point B difference."""
    import torch

    from radiacuda_b200 import rad
    import models as MD

    P = MD.magnet_array_points()

    def run(R, sync):
        h = MD.magnet_array(R)
        ts, B = [], None
        for r in range(reps + 1):
            sync()
            t0 = time.perf_counter()
            R.Solve(h, 1e-10, 1000, 4)
            B = R.Fld(h, "b", P.tolist())
            sync()
            if r:
                ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), np.array(B)

    t_ours, B_ours = run(rad, torch.cuda.synchronize)
    res = {"model": "magnet array 4x4 blocks, 3x3x3 subdivision (432 cuboids), anisotropic linear",
           "points": int(P.shape[0]), "ours_s": round(t_ours, 5)}
    R = _ref_module()
    if R is not None:
        t_ref, B_ref = run(R, lambda: None)
        res.update({"reference_cpu_s": round(t_ref, 4), "reference_cores": 1, "measured": True,
                    "ratio_reference_over_ours": round(t_ref / t_ours, 1),
                    "b_rel_err_vs_reference": b_errors(B_ours, B_ref)})
    return res


def c2_step(reps=2):
    """The saturating iron dipole: a C-yoke of 4,000 cuboids with two mirror
    planes (4 images each), MatSatIsoFrm([20000,2],[0.1,2],[0.1,2]), a
    racetrack coil of 10,000 A turns placed without symmetry; Solve to
    1e-5 (method 4) and B on the 100^3 grid in the gap (1e6 points).  Ours
    end to end through the public API (median of `reps` after a warm-up);
    beside it the reference CPU module on bounded samples, scaled and
    labelled extrapolated: assembly of a 1,000-cuboid version of the yoke
    (1 core, by n^2), its method-4 solve (1 core, by n^2 per iteration at the
    same iteration count) and Fld at 300 of the points (1 core, by the
    point count)."""
    import torch

    from radiacuda_b200 import rad
    import models as MD

    P = MD.iron_dipole_points(100)
    h = MD.iron_dipole(rad, n_target=4000)
    ts, st, parts = [], None, {}
    for r in range(reps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        im = rad.RlxPre(h)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        st = rad.RlxAuto(im, 1e-5, 5000, 4)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        rad.Fld(h, "b", P)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        rad.UtiDel(im)
        if r:
            ts.append(t3 - t0)
            parts = {"assembly": round(t1 - t0, 4), "relax": round(t2 - t1, 4), "field": round(t3 - t2, 4)}
    res = {"model": "iron dipole, 4,000 cuboids x 4 images, saturating, racetrack coil", "points": int(P.shape[0]),
           "ours_s": round(float(np.median(ts)), 4), "ours_parts_s": parts, "status": [float(x) for x in st]}
    R = _ref_module()
    if R is not None:
        hs = MD.iron_dipole(R, n_target=1000)
        t0 = time.perf_counter()
        ims = R.RlxPre(hs)
        t1 = time.perf_counter()
        sts = R.RlxAuto(ims, 1e-5, 5000, 4)
        t2 = time.perf_counter()
        from radiacuda_b200 import model
        n_small = len(model.pack_interaction(rad._objs, MD.iron_dipole(rad, n_target=1000), 0, tuple(rad._rand)).leaves)
        n_full = len(model.pack_interaction(rad._objs, MD.iron_dipole(rad, n_target=4000), 0, tuple(rad._rand)).leaves)
        hf = MD.iron_dipole(R, n_target=4000)
        Ps = P[np.random.default_rng(3).choice(P.shape[0], 300, replace=False)]
        t3 = time.perf_counter()
        R.Fld(hf, "b", Ps.tolist())
        t4 = time.perf_counter()
        scale = (float(n_full) / max(n_small, 1)) ** 2
        asm = (t1 - t0) * scale
        rlx = (t2 - t1) / max(sts[3], 1) * scale * max(st[3], 1)
        fld = (t4 - t3) * P.shape[0] / Ps.shape[0]
        res["reference_cpu"] = {"value_s": round(asm + rlx + fld, 1), "extrapolated": True, "cores": 1,
                                "parts_s": {"assembly": round(asm, 1), "relax": round(rlx, 1), "field": round(fld, 1)},
                                "sample": (f"RlxPre + RlxAuto(method 4) of the yoke at {n_small} cuboids "
                                           f"({t1 - t0:.2f} s + {t2 - t1:.2f} s, {int(sts[3])} iterations), scaled by "
                                           f"({n_full}/{n_small})^2 and our iteration count; Fld at 300 points "
                                           f"({t4 - t3:.2f} s) scaled to 1e6")}
    return res


def relax_matvec_timing():
    """The relaxation's FP32 matvec streamed from HBM, through the public API
    (rad.RlxPre with FP32 storage, rad.RlxAuto method 4: Jacobi steps with
    Anderson mixing) on the 20 x 20 magnet array: 400 blocks of 10 mm,
    anisotropic MatLin, 3x3x3 subdivision, so 10,800 cuboids, N3 = 32,400 and
    an FP32 matrix of 4.2 GB, far larger than L2.  Every iteration reads N
    once, 4 N3^2 algorithmic bytes.  The marginal time per iteration between
    runs of 20 and 60 iterations (the fastest of three each) removes the fixed
    cost of the call; the host round trip of the misfit and the Anderson
    vector work stay in it."""
    from radiacuda_b200 import _native, rad
    import models as MD

    L = _native.lib()
    h = MD.magnet_array(rad, nside=20, div=3)
    im = rad.RlxPre(h)
    n3 = 3 * 20 * 20 * 27
    rad.RlxAuto(im, 1e-30, 3, 4)
    L.radb200_device_sync()
    t, its = {}, {}
    for k in (20, 60):
        best = float("inf")
        for _ in range(3):  # the fastest of three: host stalls on a shared machine only add time
            t0 = time.perf_counter()
            st = rad.RlxAuto(im, 1e-30, k, 4, "ZeroM->False")
            L.radb200_device_sync()
            best = min(best, time.perf_counter() - t0)
        t[k], its[k] = best, int(st[3])
    rad.UtiDel(im)
    per_iter = 4.0 * n3 * n3
    marginal = (t[60] - t[20]) / max(its[60] - its[20], 1)
    if marginal <= 0.0:
        marginal = t[60] / max(its[60], 1)
    hbm = float(_peaks().get("hbm_gbs", 6650.0))
    gbs = per_iter / marginal / 1e9
    return {"model": "magnet array 20x20 blocks, 3x3x3 subdivision (10,800 cuboids)", "n3": n3,
            "matrix_bytes": per_iter, "iterations": its, "seconds": {str(k): round(v, 4) for k, v in t.items()},
            "ms_per_iteration_marginal": round(1e3 * marginal, 4),
            "ms_per_iteration_avg60": round(1e3 * t[60] / max(its[60], 1), 4),
            "achieved_gbs": round(gbs, 1), "hbm_peak_gbs": hbm, "frac": round(gbs / hbm, 4),
            "peak_source": "measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in _peaks()
            else "fallback 6650 GB/s"}


def fldint_timing(reps=3):
    """Field integrals through the public API (rad.FldInt: host packing,
    device quadrature, host result) on the relaxed planar undulator
    (2 x 40 blocks 50x10x5 mm, 2x2x2 subdivision, 640 elements) along its
    axis: the infinite first field integral and the finite one over +-150 mm,
    at PrcBInt 1e-3 (the reference's default) and 1e-6.  Median wall time of
    `reps` calls after one warm-up; beside it the reference CPU module's
    FldInt on the same relaxed model (when oracle/_ref is present) and the
    largest difference between the two."""
    import torch

    from radiacuda_b200 import rad
    import models as MD

    p1, p2 = [0.137, 0.091, -150.3], [0.137, 0.091, 149.9]
    lines = [("inf", 1e-3), ("inf", 1e-6), ("fin", 1e-3), ("fin", 1e-6)]

    def run(R, sync):
        h = MD.undulator(R, nper_row=40, div=2)[0]
        R.Solve(h, 1e-10, 1000, 4)
        out = {}
        for mode, prc in lines:
            R.FldCmpCrt(1e-4, 1e-3, prc, 1.0, 1e-5, 1e-5)
            ts, v = [], None
            for r in range(reps + 1):
                sync()
                t0 = time.perf_counter()
                v = R.FldInt(h, mode, "ib", p1, p2)
                sync()
                if r:
                    ts.append(time.perf_counter() - t0)
            out[f"{mode}_{prc:.0e}"] = (float(np.median(ts)), v)
        R.FldCmpCrt(1e-4, 1e-3, 1e-3, 1.0, 1e-5, 1e-5)
        return out

    ours = run(rad, torch.cuda.synchronize)
    res = {"model": "undulator_640 (relaxed)", "line": [p1, p2], "id": "ib",
           "ours_s": {k: round(t, 5) for k, (t, _) in ours.items()}}
    R = _ref_module()
    if R is not None:
        ref = run(R, lambda: None)
        res["reference_cpu_s"] = {k: round(t, 5) for k, (t, _) in ref.items()}
        res["max_abs_diff_Tmm"] = {k: float(np.abs(np.array(ours[k][1]) - np.array(ref[k][1])).max()) for k in ours}
    return res


def trajectory_timing(reps=3):
    """Electron trajectories through the public API (rad.FldPtcTrj) in the
    relaxed iron dipole (about 360 saturating cuboids with 4 images each, a
    racetrack coil): one 0.3 GeV trajectory through the gap over +-200 mm at
    401 points (default fixed-step Runge-Kutta: 1,600 field evaluations in
    sequence), and a batch of 1,024 trajectories (one CTA each).  Median wall
    time of `reps` after one warm-up; the reference CPU module's FldPtcTrj on
    the same relaxed model beside it, with the largest difference."""
    import torch

    from radiacuda_b200 import rad
    import models as MD

    init, lim, npt = [0.3, 0.0, 0.7, 0.0], [-200.13, 200.31], 401
    rng = np.random.default_rng(2)
    batch = np.column_stack([rng.uniform(-10, 10, 1024), rng.normal(0, 2e-3, 1024), rng.uniform(-8, 8, 1024),
                             rng.normal(0, 2e-3, 1024)])

    def timed(f, sync):
        ts, v = [], None
        for r in range(reps + 1):
            sync()
            t0 = time.perf_counter()
            v = f()
            sync()
            if r:
                ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), v

    h = MD.iron_dipole(rad, n_target=300)
    rad.Solve(h, 1e-7, 3000, 4)
    t1, ours = timed(lambda: rad.FldPtcTrj(h, 0.3, init, lim, npt), torch.cuda.synchronize)
    tb, _ = timed(lambda: rad.FldPtcTrj(h, 0.3, batch, lim, npt), torch.cuda.synchronize)
    res = {"model": "iron_dipole_300 (relaxed)", "energy_GeV": 0.3, "points": npt,
           "ours_s": {"one": round(t1, 5), "batch_1024": round(tb, 5)},
           "trajectories_per_s_batch": round(1024 / tb, 1)}
    R = _ref_module()
    if R is not None:
        hr = MD.iron_dipole(R, n_target=300)
        R.Solve(hr, 1e-7, 3000, 4)
        tr, ref = timed(lambda: R.FldPtcTrj(hr, 0.3, init, lim, npt), lambda: None)
        res["reference_cpu_s"] = {"one": round(tr, 5)}
        res["max_abs_diff"] = float(np.abs(np.array(ours) - np.array(ref)).max())
    return res


# dram__bytes_read.sum + dram__bytes_write.sum over the algorithmic bytes of the
# trailing-update kernel, from ncu captures of a 9,000^2 LU: 561 MB / 611 MB with
# TF32 operands, 475 MB / 515.7 MB with FP16 operands
TC_TRAFFIC_OVER_ALGORITHMIC = {"tf32": 0.92, "f16": 0.92}


# FP64 operations of one (point, tetrahedron) term of the vertex/edge form
# (tet_fast in csrc/formulas.cuh), counting an add/mul/compare as 1, an FMA
# as 2 and each elementary function by the cost of a standard implementation
# (sqrt, div 8; log1p 20; atan2 30): 4 vertex vectors and norms (4 x 16),
# 6 edge dot products (6 x 5), 6 edge logarithms with their accumulation
# (6 x 40), 4 solid angles with theirs (4 x 51), final scaling (3).
FIELD_OPS_PER_TET = 4 * 16 + 6 * 5 + 6 * 40 + 4 * 51 + 3

# Instructions the FP32 field kernel issues per (point, tetrahedron) pair,
# from ncu's smsp__inst_executed.sum x 32 / pairs on the 20,000-point,
# 20,000-tetrahedron case (tests/profile_cases.py field --precision single), and
# their split over the pipes.  The kernel is issue-bound: its roofline is the
# SMs' issue rate, 4 warp-instructions (128 thread-instructions) per clock
# per SM, divided by these instructions per pair.
FIELD_INST_PER_PAIR = 793
FIELD_INST_MIX = {"fma": 329, "alu": 157, "fp64": 81, "lsu": 60, "xu": 50}
B200_SMS = 148


def field_roofline(pairs_per_s, op_tflops, fp32_peak, clk):
    mhz = (clk or {}).get("sm_mhz") or 1965.0
    peak = B200_SMS * mhz * 1e6 * 128 / 1e12  # thread-instructions issued per second, 1e12
    ach = pairs_per_s * FIELD_INST_PER_PAIR / 1e12
    return {"kernel": "field_tet_kernel<float> (FP32 terms)", "bound": "issue",
            "achieved": round(ach, 3), "peak": round(peak, 3), "unit": "T instructions/s", "frac": round(ach / peak, 4),
            "peak_source": f"{B200_SMS} SMs x 128 thread-instructions per clock at the median SM clock sampled "
                           f"during the timed steps ({mhz:.0f} MHz)",
            "algorithmic": f"{FIELD_INST_PER_PAIR} instructions per (point, tetrahedron), ncu-counted "
                           f"(per pipe: {FIELD_INST_MIX})",
            "pairs_per_s": round(pairs_per_s, 1),
            "op_model": {"achieved_tflops": round(op_tflops, 3), "fp32_fma_peak_tflops": round(fp32_peak, 3),
                         "frac": round(op_tflops / fp32_peak, 4),
                         "note": f"{FIELD_OPS_PER_TET} FP64-equivalent ops per pair with elementary functions "
                                 "weighted at standard-implementation costs"},
            "traffic": None}


# ---------------------------------------------------------------------------
# CPU baselines: the reference CPU module (oracle/_ref) on a bounded sample
# ---------------------------------------------------------------------------
def _ref_module():
    d = os.path.join(ROOT, "oracle", "_ref")
    if not os.path.isdir(d) or not any(f.startswith("radia") and f.endswith(".so") for f in os.listdir(d)):
        return None
    sys.path.insert(0, d)
    import radia
    return radia


def reference_sample(small=False):
    """Extrapolated full-workload time of the reference CPU path from a
    bounded sample: assembly per pair (1 core), dense FP64 solve (LAPACK on
    all cores, scaled by n^3), field per (point, tetrahedron) (all cores)."""
    R = _ref_module()
    if R is None:
        return None
    import models as MD
    cores = os.cpu_count() or 1
    ns = 600 if small else 1500
    t0 = time.perf_counter()
    m, body = MD.tet_mesh(R, ncell=NCELL, n_tets=ns, chi=WORKLOAD["chi"])
    t1 = time.perf_counter()
    R.RlxPre(m)
    t_asm = time.perf_counter() - t1
    n_full = WORKLOAD["n_tets"]
    asm_full = t_asm * (n_full / ns) ** 2
    # LAPACK dgesv timed at a size where it already runs at its large-matrix rate
    n3s = 4000 if small else 8000
    A = np.random.default_rng(0).standard_normal((n3s, n3s)) + n3s * np.eye(n3s)
    b = np.ones(n3s)
    t2 = time.perf_counter()
    np.linalg.solve(A, b)
    t_lu = time.perf_counter() - t2
    lu_full = t_lu * (3 * n_full / n3s) ** 3
    npts = 400 if small else 2000
    # field: per point cost of the full model on one core, times the full point count / cores
    mm, _ = MD.tet_mesh(R, ncell=NCELL, n_tets=n_full, chi=WORKLOAD["chi"])
    P = MD.tet_mesh_points(npts, ncell=NCELL, seed=11)
    t3 = time.perf_counter()
    R.Fld(mm, "b", P.tolist())
    t_f = time.perf_counter() - t3
    fld_full = t_f * WORKLOAD["n_points"] / npts / cores
    total = asm_full + lu_full + fld_full
    return {"value": round(total, 2), "unit": "s", "cores": cores, "kind": "reference", "extrapolated": True,
            "sample": (f"reference CPU module: RlxPre of a {ns}-tet subset ({t_asm:.2f} s, 1 core, scaled by n^2), "
                       f"LAPACK dense solve n={n3s} ({t_lu:.2f} s, all cores, scaled by n^3), Fld of {npts} points on the "
                       f"full model ({t_f:.2f} s, 1 core, scaled to 1e6 points over {cores} cores)"),
            "parts_s": {"assembly": round(asm_full, 2), "solve": round(lu_full, 2), "field": round(fld_full, 2)}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison step (profiling runs)")
    ap.add_argument("--profile", action="store_true",
                    help="launch-list run: skip the end-to-end and CPU-baseline legs (keeps the launch count small)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", 1))
    rank = int(os.environ.get("RANK", 0))
    if args.impl == "reference":
        if rank != 0:
            return
        times = []
        last = None
        for i in range(args.warmup + args.steps):
            r = reference_sample(small=True)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference CPU module (oracle/_ref) not built"}))
                return
            if i >= args.warmup:
                times.append(r["value"])
                last = r
        v = float(np.mean(times))
        out = {"metric": METRIC, "value": round(v, 2), "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(1e3 * v, 1), "higher_is_better": False, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
               "config": dict(WORKLOAD, parallelism="cpu"),
               "cpu_baseline": {"value": round(v, 2), "unit": "s", "cores": last["cores"], "kind": "reference",
                                "extrapolated": True, "sample": last["sample"]},
               "e2e": {"value": round(v, 2), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    res = run_ours(args, rank, world)
    if not args.profile:
        res["adjoint"] = adjoint_ratio()
        res["relax_matvec"] = relax_matvec_timing()
        res["fldint"] = fldint_timing()
        res["trajectory"] = trajectory_timing()
        res["c1_end_to_end"] = c1_anchor()
        res["c2_end_to_end"] = c2_step()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = reference_sample()
        res["cpu_baseline"] = cb if cb is not None else {"value": None, "unavailable": "oracle/_ref missing"}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
