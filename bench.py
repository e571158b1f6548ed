#!/usr/bin/env python
"""Benchmark: DOF-stage updates/s of the DGSEM tendency + IMEX time stepping.

Workload (one GPU): 3-D Euler with gravity, rising warm bubble in a
10 km x 10 km x 10 km box, 16 x 16 x 16 hexahedra, N = 4 (125 LGL nodes per
element, 2,560,000 DOFs), FP64; constant-theta hydrostatic background
(theta0 = 300 K, g = 9.81), +2 K Gaussian theta bubble of 2 km radius 2 km
above ground; periodic laterally, reflective walls top/bottom; entropy-
conservative flux-differencing volume term with Rusanov surface flux; IMEX
ARK23 (split_rhs = false) with the vertical linear acoustics implicit through
the batched banded column solve.  One step = one ARK23 step = 3 stages; one
DOF-stage = one conserved variable at one node through one stage.  Inputs are
synthetic (seeded, built on the host), no dataset.

--scheme lsrk54   the same bubble stepped fully explicitly by LSRK54 (5 stages
                  per step, each one tendency launch with the register update
                  in its epilogue) instead of IMEX ARK23

--impl ours       the CUDA library through the C ABI (default)
--impl reference  the reference's CPU algorithm: the C++ oracle port (the
                  Julia reference cannot run on this image), all host cores,
                  on a horizontal sub-sample of the same workload

Prints one JSON line (rank 0).  N > 1 GPUs: independent replicas, one per
rank (the served/batched instances are independent; no data-path
collective), scaling "weak", time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic FP64 flops per DOF-stage of the flux-differencing tendency
# (EC volume flux, Rusanov surface flux), from the oracle's instrumented
# counter: python oracle/count_flops.py
FLOPS_PER_DOF_STAGE = {"bubble_3d_N4_ec_rusanov": 602.8, "bubble_3d_N7_ec_rusanov": 896.2,
                       "bubble_3d_N4_linear_weak_z": 22.4, "bubble_3d_N7_linear_weak_z": 25.1,
                       "sphere_N5_ec_rusanov": 736.5, "sphere_N5_linear_weak_z": 22.9}
L2_BYTES = 126 * 2 ** 20


def load_pkg():
    from __graft_entry__ import _load_package
    return _load_package()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.p = None
        self.path = os.path.join("/tmp", f"atb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.f.close()

    def summary(self):
        if self.p is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


SCHEME_STAGES = {"ark23": 3, "lsrk54": 5}


def build_case(precision="fp64", K=16, scheme="ark23"):
    """The rising bubble: IMEX ARK23 with the vertical acoustics implicit, or
    the fully explicit LSRK54 run of the same problem at its smaller dt."""
    load_pkg()
    from atum_b200 import workloads as P
    return P.bubble_3d(N=4, K=K, imex=(scheme == "ark23"), steps=200, precision=precision)


def make_solver(A, case, q, scheme):
    if scheme == "ark23":
        return A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
    return A.LSRK54(case.dg, q, case.dt)


def make_oracle_solver(orc, case, q, scheme):
    dg = orc.DGSEM(case.dg)
    if scheme == "ark23":
        return orc.ARK23(dg, orc.DGSEM(case.lindg), q, case.dt, split_rhs=False)
    return orc.LSRK54(dg, q, case.dt)


def scheme_label(scheme):
    return ("IMEX ARK23 split_rhs=false, vertical banded solve" if scheme == "ark23"
            else "explicit LSRK54 (Carpenter-Kennedy 5-stage)")


def workload_config(scheme, precision="fp64"):
    """The ``config`` dict both arms print for the rising-bubble workload
    (identical, so the two lines name the same workload)."""
    return {"workload": "3-D Euler-gravity rising bubble, 16^3 hexahedra, N=4 (2,560,000 DOFs), EC volume + "
                        "Rusanov surface flux, " + scheme_label(scheme),
            "dofs": 2560000, "stages_per_step": SCHEME_STAGES[scheme], "precision": precision,
            "l2": "working set ~0.21 GB > 126 MB L2 (no flush)"}


def dist_init():
    """One process per GPU (torchrun's RANK / WORLD_SIZE / MASTER_*): NCCL with
    GPUs, gloo without (the CPU tests of this plumbing)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
        return dist, int(os.environ.get("RANK", "0")), world
    return None, 0, 1


def max_over_ranks(x: float, dist) -> float:
    """The largest of every rank's value (device times: the job takes as long
    as its slowest rank)."""
    if dist is None:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, dist) -> float:
    """The sum of every rank's value (work done by independent replicas)."""
    if dist is None:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def instance_seeds(n_inst: int, rank: int):
    """Seeds of one rank's independent instances (replicas: ranks share no
    instance, so no data-path collective is needed)."""
    return [1000 * (rank + 1) + i for i in range(n_inst)]


# ----------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's algorithm on the host cores (the oracle port, all
    threads): each step one step of the full workload when the requested
    steps fit in about three minutes, else of the 4x4x16-element horizontal
    sub-sample (same columns, physics and dt)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as orc
    load_pkg()
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    case = build_case(scheme=args.scheme)
    q = case.q0.copy()
    s = make_oracle_solver(orc, case, q, args.scheme)
    t0 = time.perf_counter()
    s.step(q, 1)
    t1 = time.perf_counter() - t0
    if (args.steps + args.warmup) * t1 > 180.0:
        case = build_case_sample(args.scheme)
        q = case.q0.copy()
        s = make_oracle_solver(orc, case, q, args.scheme)
        Kd = case.dg.grid.Kd
        sample = (f"{Kd[0]}x{Kd[1]}x{Kd[2]} elements (a horizontal sub-sample of the 16x16x16 workload, same "
                  f"columns), {q.size} DOFs, {args.scheme.upper()} steps")
    else:
        sample = f"the full 16x16x16-element workload, {q.size} DOFs, {args.scheme.upper()} steps"
    dofs = q.size
    s.step(q, args.warmup)
    t0 = time.perf_counter()
    s.step(q, args.steps)
    T = time.perf_counter() - t0
    v = dofs * SCHEME_STAGES[args.scheme] * args.steps / T
    line = {"metric": "DOF-stage updates/s", "value": v, "unit": "DOF-stage/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": T / args.steps * 1e3, "higher_is_better": True,
            "impl": "reference", "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.scheme), "parallelism": f"{threads} host threads",
            "cpu_baseline": {"value": v, "unit": "DOF-stage/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "vs_baseline": None}
    print(json.dumps(line), flush=True)
    return 0


def build_case_sample(scheme="ark23"):
    """Horizontal sub-sample of the benchmark workload: 4x4 of the 16x16
    element columns at full height, identical spacing, physics and dt."""
    import numpy as np
    load_pkg()
    from atum_b200 import workloads as P
    import atum_b200 as A
    full = build_case(scheme=scheme)
    L = 10e3
    K = 16
    v = np.array([L * i / K for i in range(K + 1)])
    vh = v[:5]
    law = full.dg.law
    cell = full.dg.grid.cell
    grid = A.brickgrid(cell, (vh, vh, v), periodic=(True, True, False), ordering="stacked")
    dg = A.DGSEM(law=law, grid=grid, volume_form=full.dg.volume_form, surface_numericalflux=A.RusanovFlux())
    aux = dg.auxstate_host()
    lin = A.DGSEM(law=A.LinearEulerGravityLaw(law), grid=grid, surface_numericalflux=A.RusanovFlux(), auxstate=aux,
                  directions=(3,))
    # same initial condition formula on the sub-grid
    x = grid.points()
    cv, g = 719.0, law.gamma
    cp, R = g * cv, g * cv - cv
    r = np.sqrt((x[0] - L / 2) ** 2 + (x[1] - L / 2) ** 2 + (x[2] - 2000.0) ** 2)
    theta = 300.0 + 2.0 * np.exp(-(r / 2000.0) ** 2)
    pi_ex = 1 - law.grav / (cp * 300.0) * x[2]
    p = 1e5 * pi_ex ** (cp / R)
    rho = p / (R * theta * pi_ex)
    z = np.zeros_like(rho)
    q0 = np.ascontiguousarray(np.stack([rho, z, z, z, law.energy(rho, [z, z, z], p, aux[0])]))
    if scheme != "ark23":
        return P.Case("bubble_3d_sample", dg, q0, full.dt, full.timeend)
    return P.Case("bubble_3d_sample", dg, q0, full.dt, full.timeend, solver="ARK23", lindg=lin, split_rhs=False,
                  adjust_final=False)


def _time_steps(s, q, min_s, max_steps):
    """Steps s until at least min_s seconds have passed (or max_steps); the
    number of steps and the seconds they took."""
    n, t0 = 0, time.perf_counter()
    while n < max_steps:
        s.step(q, 1)
        n += 1
        if time.perf_counter() - t0 >= min_s:
            break
    return n, time.perf_counter() - t0


def cpu_baseline_sample(scheme="ark23", min_s=10.0):
    """Oracle port on the host cores: all cores on the full workload, and one
    core on the 4x4x16-element horizontal sub-sample, each timed for about
    min_s seconds after one warm-up step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as orc
    stages = SCHEME_STAGES[scheme]
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    full = build_case(scheme=scheme)
    q = full.q0.copy()
    s = make_oracle_solver(orc, full, q, scheme)
    s.step(q, 1)
    n, T = _time_steps(s, q, min_s, 200)
    line = {"value": q.size * stages * n / T, "unit": "DOF-stage/s", "cores": threads, "kind": "port",
            "sample": f"{n} {scheme.upper()} steps of the full 16x16x16-element workload ({q.size} DOFs), "
                      f"{threads} threads, {T:.1f} s"}
    del s, q
    orc.set_threads(1)
    sub = build_case_sample(scheme)
    q1 = sub.q0.copy()
    s1 = make_oracle_solver(orc, sub, q1, scheme)
    s1.step(q1, 1)
    n1, T1 = _time_steps(s1, q1, min_s / 2, 200)
    line["one_core"] = {"value": q1.size * stages * n1 / T1, "unit": "DOF-stage/s", "cores": 1,
                        "sample": f"{n1} {scheme.upper()} steps of a 4x4x16-element horizontal sub-sample "
                                  f"({q1.size} DOFs, same columns, physics and dt), 1 thread, {T1:.1f} s"}
    orc.set_threads(threads)
    return line


# ---------------------------------------------------------------- our arm
def run_ours(args):
    import numpy as np
    import torch

    dist, rank, world = dist_init()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    A = load_pkg()
    from atum_b200 import _lib

    scheme = args.scheme
    stages = SCHEME_STAGES[scheme]
    case = build_case(args.precision, scheme=scheme)
    dofs = case.q0.size
    q = torch.as_tensor(case.q0, device="cuda").contiguous()
    # launch shapes picked by the library's autotuner (results do not depend on
    # them), or the explicit operator's given (a profiler's replays perturb the
    # autotuner's timings)
    if args.elements_per_cta:
        A.batch.set_launch(case.dg, args.elements_per_cta)
        tuned = {"tendency": args.elements_per_cta}
    else:
        tuned = {"tendency": A.batch.autotune(case.dg, q)}
    if scheme == "ark23":
        tuned["tendency_linear"] = A.batch.autotune(case.lindg, q)
    solver = make_solver(A, case, q, scheme)
    L = _lib.lib()
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    solver.step(q, args.warmup)
    barrier()
    n0 = _lib.C.c_long()
    L.atb_launch_count(_lib.C.byref(n0))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        barrier()
        ev0.record(stream)
        solver.step(q, args.steps)
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    n1 = _lib.C.c_long()
    L.atb_launch_count(_lib.C.byref(n1))
    # per-kernel times from a second pass with the library's per-launch CUDA
    # events (kept out of the headline timing above)
    kprof = max(3, min(args.steps, 30))
    _lib.check(L.atb_profile_reset())
    _lib.check(L.atb_profile_enable(1))
    solver.step(q, kprof)
    barrier()
    _lib.check(L.atb_profile_enable(0))
    prof = {"steps": kprof}
    for k, name in enumerate(("tendency", "tendency_linear", "band_solve", "combine", "reduce")):
        nl, tm = _lib.C.c_long(), _lib.C.c_double()
        _lib.check(L.atb_profile_read(k, _lib.C.byref(nl), _lib.C.byref(tm)))
        prof[name] = {"launches": nl.value, "ms": tm.value}
    ms = max_over_ranks(ms, dist)
    assert torch.isfinite(q).all(), "non-finite state after the timed steps"

    # ------------------------------------------------------------- e2e
    # Through the public API with host buffers: every step copies the state
    # from pinned host memory to the device and the result back.
    qh = torch.empty(case.q0.shape, dtype=torch.float64, pin_memory=True)
    qh.copy_(torch.as_tensor(case.q0))
    qd = torch.empty_like(q)
    s2 = make_solver(A, case, qd, scheme)
    ke = max(3, min(args.steps, 50))
    qd.copy_(qh, non_blocking=True)
    s2.step(qd, 1)
    qh.copy_(qd, non_blocking=True)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(ke):
        qd.copy_(qh, non_blocking=True)
        s2.step(qd, 1)
        qh.copy_(qd, non_blocking=True)
    e1.record(stream)
    barrier()
    ms_e2e = e0.elapsed_time(e1)
    ms_e2e = max_over_ranks(ms_e2e, dist)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    value = world * dofs * stages * args.steps / (ms * 1e-3)
    e2e = world * dofs * stages * ke / (ms_e2e * 1e-3)
    tend = prof["tendency"]
    avg_ms = tend["ms"] / max(1, tend["launches"])
    # the stage kernel: explicit EC tendency fused with the linear vertical
    # operator when the solver fuses them (no separate linear launches)
    fused = scheme == "ark23" and prof["tendency_linear"]["launches"] == 0
    flops_dof = FLOPS_PER_DOF_STAGE["bubble_3d_N4_ec_rusanov"]
    if fused:
        flops_dof += FLOPS_PER_DOF_STAGE["bubble_3d_N4_linear_weak_z"]
    flops_launch = flops_dof * dofs
    tflops = flops_launch / (avg_ms * 1e-3) / 1e12
    peak_fp64 = _lib.C.c_double()
    _lib.check(L.atb_probe_fp64_peak(_lib.C.byref(peak_fp64), _lib.stream_ptr()))
    peaks, kind = measured_peaks()
    # algorithmic bytes per launch: fused stage kernel, averaged over the three
    # stages: Q (5) and aux (6) read; accumulators 15 written (stage 1), 10 read
    # + 10 written (stage 2), 5 read + 5 written (stage 3) -> 26 x 8 B per node.
    # LSRK54 stage kernel (tendency + register update in its epilogue): Q (5)
    # and Phi (1) read, dQ read (5, stages 2-5), dQ and Q written (10) -> 20 on
    # average.  Unfused ARK explicit tendency: Q (5), Phi (1) read, N(Q) (5)
    # written.
    bytes_launch = (26 if fused else 20 if scheme == "lsrk54" else 11) * 8 * dofs // 5
    line = {
        "metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64-state/f32-flux",
        "data": "synthetic",
        "config": workload_config(scheme, args.precision),
        "parallelism": f"replicas x{world}" if world > 1 else "1 GPU", "elements_per_cta": tuned,
        "e2e": {"value": e2e, "unit": "DOF-stage/s", "h2d_bytes_per_step": dofs * 8, "d2h_bytes_per_step": dofs * 8,
                "steps": ke},
        "gpu_launches": int(n1.value - n0.value),
        "roofline": {"bound": "fp64",
                     "kernel": ("tendency_kernel<EulerGravity,3,EC,Nq=5,fused> (ARK23 stage: EC tendency + linear "
                                "vertical operator)") if fused else
                               ("tendency_kernel<EulerGravity,3,EC,Nq=5> (LSRK54 stage: tendency + register "
                                "update)" if scheme == "lsrk54" else
                                "tendency_kernel<EulerGravity,3,EC,Nq=5> (explicit stage tendency)"),
                     "flops_per_dof_stage": flops_dof,
                     "achieved": tflops, "peak": peak_fp64.value, "unit": "TFLOP/s",
                     "frac": tflops / peak_fp64.value if peak_fp64.value > 0 else None,
                     "peak_source": "measured in this run: FP64 FMA probe (atb_probe_fp64_peak)",
                     "flops_per_launch": flops_launch, "avg_launch_ms": avg_ms,
                     "traffic": profiled_traffic(PROFILE_FUSED if fused else PROFILE_TEND)
                     if args.precision == "fp64" else None,
                     "traffic_unit": "bytes per launch (dram read + write, one ncu capture)",
                     "traffic_source": PROFILE_FUSED if fused else PROFILE_TEND,
                     "hbm_view": {"bytes_per_launch": bytes_launch,
                                  "achieved_gbs": bytes_launch / (avg_ms * 1e-3) / 1e9,
                                  "peak_gbs": peaks["hbm_gbs"], "peak_kind": kind}},
        "kernels": prof,
        "clocks": clk.summary(),
    }
    if world == 1 and args.precision == "fp64" and not args.no_precision_pair:
        line["fp32flux"] = precision_pair(A, args, scheme, value)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(scheme)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def precision_pair(A, args, scheme, value_fp64):
    """The FP32-flux / FP64-state form on the same inputs: its throughput
    (timed like the headline, inputs resident), and its error after
    ``args.steps`` steps from the same initial state against the FP64 path --
    relative L2 (MJ-weighted) and L-infinity per component -- plus the mass
    drift of both forms (the box is closed: periodic sides, walls at top and
    bottom)."""
    import numpy as np
    import torch

    stream = torch.cuda.current_stream()
    c64 = build_case("fp64", scheme=scheme)
    c32 = build_case("fp32flux", scheme=scheme)
    q = torch.as_tensor(c32.q0, device="cuda").contiguous()
    A.batch.autotune(c32.dg, q)
    if scheme == "ark23":
        A.batch.autotune(c32.lindg, q)
    s32 = make_solver(A, c32, q, scheme)
    s32.step(q, args.warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s32.step(q, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    v32 = c32.q0.size * SCHEME_STAGES[scheme] * args.steps / (ms * 1e-3)
    # accuracy: both forms from the same initial state, the same steps
    qa = torch.as_tensor(c64.q0, device="cuda").contiguous()
    qb = torch.as_tensor(c32.q0, device="cuda").contiguous()
    make_solver(A, c64, qa, scheme).step(qa, args.steps)
    make_solver(A, c32, qb, scheme).step(qb, args.steps)
    torch.cuda.synchronize()
    diff = (qb - qa).contiguous()
    rel_l2 = A.weightednorm(c64.dg, diff) / A.weightednorm(c64.dg, qa)
    ha, hb, h0 = qa.cpu().numpy(), qb.cpu().numpy(), c64.q0
    linf = [float(np.max(np.abs(hb[c] - ha[c])) / np.max(np.abs(ha[c]))) for c in range(ha.shape[0])]
    mj = c64.dg.MJ
    m0 = float(np.sum(mj * h0[0]))
    return {"value": v32, "unit": "DOF-stage/s", "ms_per_step": ms / args.steps, "steps": args.steps,
            "speedup_vs_fp64": v32 / value_fp64, "rel_l2_vs_fp64": rel_l2, "rel_linf_vs_fp64_per_component": linf,
            "steps_compared": args.steps,
            "mass_drift_fp64": abs(float(np.sum(mj * ha[0])) - m0) / abs(m0),
            "mass_drift_fp32flux": abs(float(np.sum(mj * hb[0])) - m0) / abs(m0)}


PROFILE_TEND = "profiles/tendency_eg3_ec_nq5_bubble16.md"
PROFILE_FUSED = "profiles/tendency_eg3_ec_nq5_fused_bubble16.md"


# ------------------------------------------------------------ serving stream
def run_serve(args):
    """Seeded Poisson stream of requests served by continuous batching: 2-D
    Euler isentropic vortices (periodic [-5,5]^2, 16^2..128^2 elements) and
    3-D Euler-gravity rising bubbles (8^3..32^3 elements), orders N uniform in
    2..7, FP32 flux / FP64 state, LSRK54 at CFL 0.3, end times uniform in
    0.5..5 flow-through times multiplied by --time-scale (a full flow-through
    takes thousands of steps per request; the scale keeps the run to about a
    minute).  Requests are admitted under an HBM budget and packed by (law, N).
    Reports throughput, p50/p99 latency, and the relative L2 error of a sample
    of requests against the same request stepped alone by the FP64 path."""
    import numpy as np
    import torch

    dist, rank, world = dist_init()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    A = load_pkg()
    load_pkg()
    from atum_b200 import workloads as P

    vortex_K = list(range(16, 129, 16))
    bubble_K = [8, 16, 24, 32]
    cache = {}

    def spec(kind, K, N, precision):
        """(case, flow-through time, device builder of the initial state and
        aux fields); the host case supplies the operator spec and dt only."""
        key = (kind, K, N, precision)
        if key not in cache:
            if kind == "vortex":
                c = P.vortex_c1(N=N, K=K, precision=precision)
                flow = 10.0 / math.sqrt(2.0)          # domain / |u|
                make = (lambda dg=c.dg: P.vortex_c1_device(dg))
            else:
                c = P.bubble_3d(N=N, K=K, imex=False, precision=precision)
                flow = 10e3 / 340.0                   # box / sound speed
                make = (lambda dg=c.dg: P.bubble_3d_device(dg))
            c.q0 = None  # inputs are built on the device at admission
            cache[key] = (c, flow, make)
        return cache[key]

    def stream(time_scale, seed):
        rng = np.random.default_rng(seed)
        reqs = []
        t = 0.0
        for i in range(args.requests):
            t += rng.exponential(1.0 / args.rate)
            kind = "vortex" if rng.random() < 0.5 else "bubble"
            K = int(rng.choice(vortex_K if kind == "vortex" else bubble_K))
            N = int(rng.integers(2, 8))
            c, flow, make = spec(kind, K, N, "fp32flux")
            tend = rng.uniform(0.5, 5.0) * flow * time_scale
            nsteps = max(1, int(math.ceil(tend / c.dt)))
            # the client asks for the final state's weighted norms only ...
            reqs.append(A.serving.Request(rid=i, dg=c.dg, q0=None, make=make, dt=c.dt, nsteps=nsteps,
                                          arrival=t, keep_result=True, result_mode="norms"))
        # ... except a sample whose whole state is checked against FP64
        sampled = reqs[:: max(1, len(reqs) // args.error_samples)][: args.error_samples]
        for r in sampled:
            r.result_mode = "state"
        return reqs, sampled

    srv = A.serving.Server(hbm_budget_bytes=args.hbm_budget_gb * 1e9, chunk=256, use_graphs=True,
                           pool_bytes=args.pool_gb * 1e9, result_bytes=args.result_gb * 1e9)
    reqs, sampled = stream(args.time_scale, 20261203 + rank)
    # warm-up stream (a few requests), then the measured one
    warm = [A.serving.Request(rid=-1 - j, dg=r.dg, q0=None, make=r.make, dt=r.dt, nsteps=min(r.nsteps, 4),
                              arrival=0.0, keep_result=False) for j, r in enumerate(reqs[:args.warmup])]
    srv.run(warm, realtime=False)
    with ClockSampler(torch.cuda.current_device()) as clk:
        st = srv.run(reqs, realtime=True)
    clocks = clk.summary()  # read before the next sampler reuses the file
    # the same arrivals with end times a fifth as long: an offered load one
    # B200 sustains, so latency measures serving rather than queueing
    reqs_s, _ = stream(args.time_scale / 5, 20261203 + rank)
    with ClockSampler(torch.cuda.current_device()) as clk_s:
        st_s = srv.run(reqs_s, realtime=True)
    clocks_s = clk_s.summary()
    lat_s = np.array([r.latency for r in reqs_s])
    # accuracy: a sample of requests stepped alone in FP64 from the same
    # device-built initial state
    errs = []
    for r in sampled:
        kind = "vortex" if r.dg.law.dim == 2 else "bubble"
        c64, _, make64 = spec(kind, int(round(r.dg.grid.Kd[0])), r.dg.grid.cell.N, "fp64")
        q = make64()[0]
        A.LSRK54(c64.dg, q, r.dt).step(q, r.nsteps)
        ref = q.cpu().numpy()
        MJ = c64.dg.MJ
        num = sum(float(np.sum(MJ * (r.result[s] - ref[s]) ** 2)) for s in range(ref.shape[0]))
        den = sum(float(np.sum(MJ * ref[s] ** 2)) for s in range(ref.shape[0]))
        errs.append(math.sqrt(num / den))
    srv.close()
    span = max_over_ranks(st.makespan_s, dist)
    total = sum_over_ranks(st.extra["dof_stage_updates"], dist)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    lat = np.array([r.latency for r in reqs])
    line = {
        "metric": "DOF-stage updates/s", "value": total / span, "unit": "DOF-stage/s",
        "n_gpus": world, "steps": int(sum(r.nsteps for r in reqs)), "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64-state/f32-flux", "data": "synthetic",
        "config": {"workload": "serving: Poisson stream of 2-D Euler vortices (16^2..128^2) and 3-D Euler-gravity "
                               "bubbles (8^3..32^3), N in 2..7, FP32 flux / FP64 state, LSRK54, packed by (law, N)",
                   "requests": args.requests, "rate_per_s": args.rate, "time_scale": args.time_scale,
                   "hbm_budget_gb": args.hbm_budget_gb, "pool_gb": args.pool_gb},
        "latency_s": {"p50": st.p50_latency_s, "p99": st.p99_latency_s, "mean": st.mean_latency_s,
                      "max": float(lat.max())},
        "sustainable": {"time_scale": args.time_scale / 5, "value": st_s.dof_stage_per_s, "unit": "DOF-stage/s",
                        "latency_s": {"p50": st_s.p50_latency_s, "p99": st_s.p99_latency_s,
                                      "mean": st_s.mean_latency_s, "max": float(lat_s.max())},
                        "makespan_s": st_s.makespan_s, "arrival_window_s": max(r.arrival for r in reqs_s),
                        "dof_stage_updates": st_s.extra["dof_stage_updates"],
                        "host_seconds": st_s.extra["host_seconds"], "clocks": clocks_s},
        "inputs": "built on the device at admission (grid points, aux fields, initial state)",
        "results": "per-component weighted L2 norms copied back; whole states only for the sampled requests",
        "makespan_s": st.makespan_s, "arrival_window_s": max(r.arrival for r in reqs),
        "pools": st.pools, "ticks": st.ticks,
        "host_seconds": st.extra["host_seconds"],
        "result_arena_fallbacks": st.extra.get("result_arena_fallbacks"),
        "peak_pool_bytes": st.peak_pool_bytes, "dof_stage_updates": st.extra["dof_stage_updates"],
        "rel_l2_vs_fp64": {"samples": len(errs), "max": max(errs) if errs else None,
                           "median": float(np.median(errs)) if errs else None},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------- large single instance
def run_c5(args):
    """3-D Euler-gravity on 128 x 128 x 32 hexahedra, N = 7 (1.342 G DOFs) in
    a 40 km x 40 km x 10 km box (isotropic 312.5 m elements), periodic
    laterally, reflective walls top and bottom; constant-theta hydrostatic
    background (theta0 = 300 K) with a seeded smooth theta perturbation of
    +-0.5 K (random Fourier modes of wavelengths 4-16 elements); IMEX ARK23
    (split_rhs = false, vertical acoustics through the banded column solve).
    Grid points, aux fields and the initial state are built on the device.
    The same 50 steps run with FP64 flux arithmetic and with the FP32-flux
    form; reported: both throughputs, the FP32-flux error against FP64, mass
    drift, and per-kernel times with roofline fractions."""
    import numpy as np
    import torch

    dist, rank, world = dist_init()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    A = load_pkg()
    from atum_b200 import _lib
    from atum_b200.cell import points_device
    load_pkg()
    from atum_b200 import workloads as P

    Kx, Ky, Kz = args.c5_elements
    N = 7
    steps = args.steps if args.steps is not None else 50
    Lh, H = 40e3 * Kx / 128, 10e3 * Kz / 32
    vx = np.array([Lh * i / Kx for i in range(Kx + 1)])
    vy = np.array([Lh * i / Ky for i in range(Ky + 1)])
    vz = np.array([H * i / Kz for i in range(Kz + 1)])
    cell = A.LobattoCell(N + 1, N + 1, N + 1)
    grid = A.brickgrid(cell, (vx, vy, vz), periodic=(True, True, False), ordering="stacked")
    law = A.EulerGravityLaw(3, grav=9.81, problem=A.ReflectiveWall(referencestate=P.bubble_reference))
    g = law.grav
    cv = 719.0
    cp = law.gamma * cv
    R = cp - cv
    x = points_device(grid)
    z = x[2]
    pi_ex = 1 - g / (cp * 300.0) * z
    aux = torch.zeros((law.naux,) + tuple(z.shape), dtype=torch.float64, device="cuda")
    aux[0] = g * z
    aux[3] = g
    aux[4] = 1e5 / (R * 300.0) * pi_ex ** (cv / R)
    aux[5] = 1e5 * pi_ex ** (cp / R)
    # smooth seeded theta perturbation: random modes, wavelengths 4-16 elements
    rng = np.random.default_rng(20261203)
    dth = torch.zeros_like(z)
    he = Lh / Kx
    for _ in range(24):
        lam = rng.uniform(4, 16, 3) * he
        kx = 2 * np.pi * max(1, round(Lh / lam[0])) / Lh * rng.choice([-1, 1])
        ky = 2 * np.pi * max(1, round(Lh / lam[1])) / Lh * rng.choice([-1, 1])
        kz = 2 * np.pi / lam[2]
        dth += rng.standard_normal() * torch.cos(kx * x[0] + ky * x[1] + kz * z + rng.uniform(0, 2 * np.pi))
    dth *= 0.5 / dth.abs().max()
    del x
    p = aux[5]
    rho = p / (R * (300.0 + dth) * pi_ex)
    del dth, pi_ex
    q0 = torch.zeros((5,) + tuple(z.shape), dtype=torch.float64, device="cuda")
    q0[0] = rho
    q0[4] = p / (law.gamma - 1) + rho * aux[0]
    del rho, p, z
    dofs = q0.numel()
    lin = A.LinearEulerGravityLaw(law)
    lindg = A.DGSEM(law=lin, grid=grid, surface_numericalflux=A.RusanovFlux(), auxstate=aux, directions=(3,))
    dz = A.min_node_distance(grid, dims=(3,))
    dt = 0.25 * dz / 340.0
    w = torch.as_tensor(np.asarray(cell.weights, dtype=np.float64), device="cuda")
    w3 = (w[:, None, None] * w[None, :, None] * w[None, None, :]).reshape(-1)  # node order i fastest
    L = _lib.lib()
    peak_fp64 = _lib.C.c_double()
    _lib.check(L.atb_probe_fp64_peak(_lib.C.byref(peak_fp64), _lib.stream_ptr()))
    peaks, kind = measured_peaks()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def run(precision):
        dg = A.DGSEM(law=law, grid=grid, volume_form=A.FluxDifferencingForm(A.EntropyConservativeFlux()),
                     surface_numericalflux=A.RusanovFlux(), auxstate=aux, precision=precision)
        torch.cuda.empty_cache()
        q = q0.clone()
        s = A.ARK23(dg, lindg, q, dt, split_rhs=False)
        s.step(q, args.warmup)
        q.copy_(q0)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = _lib.C.c_long()
        L.atb_launch_count(_lib.C.byref(n0))
        e0.record()
        s.step(q, steps)
        e1.record()
        barrier()
        ms = e0.elapsed_time(e1)
        n1 = _lib.C.c_long()
        L.atb_launch_count(_lib.C.byref(n1))
        # per-kernel times: a few more steps with the library's launch events
        qp = q.clone()
        _lib.check(L.atb_profile_reset())
        _lib.check(L.atb_profile_enable(1))
        s.step(qp, 3)
        barrier()
        _lib.check(L.atb_profile_enable(0))
        prof = {}
        for k, name in enumerate(("tendency", "tendency_linear", "band_solve", "combine", "reduce")):
            nl, tm = _lib.C.c_long(), _lib.C.c_double()
            _lib.check(L.atb_profile_read(k, _lib.C.byref(nl), _lib.C.byref(tm)))
            prof[name] = {"launches": nl.value, "ms": tm.value}
        del qp, s, dg
        import gc
        gc.collect()  # the operator and its spec refer to each other
        torch.cuda.empty_cache()
        return q, ms, int(n1.value - n0.value), prof

    with ClockSampler(torch.cuda.current_device()) as clk:
        q64, ms64, nl64, prof64 = run("fp64")
        q32, ms32, nl32, prof32 = run("fp32flux")
    ms64, ms32 = max_over_ranks(ms64, dist), max_over_ranks(ms32, dist)
    assert torch.isfinite(q64).all() and torch.isfinite(q32).all(), "non-finite state"

    def wnorm2(a):
        return float(sum(((a[c] ** 2) * w3[None, :]).sum() for c in range(a.shape[0])))

    rel = math.sqrt(wnorm2(q32 - q64) / wnorm2(q64))
    pert = math.sqrt(wnorm2(q32 - q64) / wnorm2(q64 - q0))
    m0 = float((q0[0] * w3[None, :]).sum())
    drift64 = abs(float((q64[0] * w3[None, :]).sum()) - m0) / m0
    drift32 = abs(float((q32[0] * w3[None, :]).sum()) - m0) / m0
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    def kernels(prof, precision):
        out = {}
        fused = prof["tendency_linear"]["launches"] == 0
        t = prof["tendency"]
        avg = t["ms"] / max(1, t["launches"])
        fl = (FLOPS_PER_DOF_STAGE["bubble_3d_N7_ec_rusanov"] +
              (FLOPS_PER_DOF_STAGE["bubble_3d_N7_linear_weak_z"] if fused else 0.0)) * dofs
        out["stage_kernel"] = {"kernel": "tendency_kernel<EulerGravity,3,%s,Nq=8%s>" %
                               ("EC" if precision == "fp64" else "EC32", ",fused" if fused else ""),
                               "avg_launch_ms": avg, "bound": "fp64", "achieved_tflops": fl / (avg * 1e-3) / 1e12,
                               "peak_tflops": peak_fp64.value,
                               "frac": fl / (avg * 1e-3) / 1e12 / peak_fp64.value}
        b = prof["band_solve"]
        if b["launches"]:
            avgb = b["ms"] / b["launches"]
            # right-hand side read, solution written, read back and rewritten
            byt = 4 * dofs * 8
            out["band_solve"] = {"kernel": "band_solve_warp_kernel<8,5> (tile-sparse warp-owned recurrence)", "avg_launch_ms": avgb, "bound": "hbm",
                                 "achieved_gbs": byt / (avgb * 1e-3) / 1e9, "peak_gbs": peaks["hbm_gbs"],
                                 "frac": byt / (avgb * 1e-3) / 1e9 / peaks["hbm_gbs"], "peak_kind": kind}
        out["launch_totals"] = prof
        return out

    v64 = world * dofs * 3 * steps / (ms64 * 1e-3)
    v32 = world * dofs * 3 * steps / (ms32 * 1e-3)
    line = {
        "metric": "DOF-stage updates/s", "value": v64, "unit": "DOF-stage/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms64 / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (built on the device)",
        "config": {"workload": f"3-D Euler-gravity, {Kx}x{Ky}x{Kz} hexahedra, N=7 ({dofs} DOFs), hydrostatic "
                               "background + seeded smooth theta' (+-0.5 K), EC volume + Rusanov surface flux, "
                               "IMEX ARK23 split_rhs=false, vertical banded solve",
                   "dofs": dofs, "stages_per_step": 3, "box_m": [Lh, Lh, H], "dt_s": dt,
                   "l2": f"working set ~{dofs * 8 * 12 / 1e9:.0f} GB >> 126 MB L2 (no flush)"},
        "gpu_launches": nl64,
        "fp32flux": {"value": v32, "ms_per_step": ms32 / steps, "gpu_launches": nl32,
                     "speedup_vs_fp64": v32 / v64,
                     "rel_l2_vs_fp64": rel, "rel_l2_vs_fp64_of_perturbation": pert},
        "mass_drift": {"fp64": drift64, "fp32flux": drift32},
        "kernels": {"fp64": kernels(prof64, "fp64"), "fp32flux": kernels(prof32, "fp32flux")},
        "clocks": clk.summary(),
        "e2e": None,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------ cubed-sphere shell
def run_sphere(args):
    """Acoustic wave on an Earth-radius cubed-sphere shell in the reference's
    own configuration (experiment/euler_gravity/acousticwave.jl: N = 5,
    KH = 10, KV = 5: 3000 curved hexahedra, 648,000 nodes, 3.24 M DOFs, 10 km
    deep), EC volume + Rusanov surface flux, IMEX ARK23 (split_rhs = false)
    with the vertical acoustics in the banded column solve (one band per
    vertical line of nodes: the columns of a sphere differ), dt = 100 (H/KV) /
    330 / N^2 (about 20 s).  Curved-element kernels: per-node metric terms, per
    face-node normals, a node-level face map."""
    import numpy as np
    import torch

    dist, rank, world = dist_init()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    A = load_pkg()
    from atum_b200 import _lib
    from atum_b200 import workloads as P

    N, KH, KV = 5, 10, 5
    steps = args.steps if args.steps is not None else 20
    t0 = time.perf_counter()
    case = P.sphere_acoustic_wave(N=N, KH=KH, KV=KV, steps=steps)
    t_setup = time.perf_counter() - t0
    dofs = case.q0.size
    L = _lib.lib()
    stream = torch.cuda.current_stream()
    q0 = torch.as_tensor(case.q0, device="cuda").contiguous()
    q = q0.clone()
    tuned = {"tendency": A.batch.autotune(case.dg, q), "tendency_linear": A.batch.autotune(case.lindg, q)}
    t0 = time.perf_counter()
    s = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
    torch.cuda.synchronize()
    t_solver = time.perf_counter() - t0

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    s.step(q, args.warmup)
    q.copy_(q0)
    barrier()
    n0 = _lib.C.c_long()
    L.atb_launch_count(_lib.C.byref(n0))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        barrier()
        e0.record(stream)
        s.step(q, steps)
        e1.record(stream)
        barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    n1 = _lib.C.c_long()
    L.atb_launch_count(_lib.C.byref(n1))
    assert torch.isfinite(q).all(), "non-finite state after the timed steps"
    _lib.check(L.atb_profile_reset())
    _lib.check(L.atb_profile_enable(1))
    qp = q.clone()
    s.step(qp, 3)
    barrier()
    _lib.check(L.atb_profile_enable(0))
    prof = {"steps": 3}
    for k, name in enumerate(("tendency", "tendency_linear", "band_solve", "combine", "reduce")):
        nl, tm = _lib.C.c_long(), _lib.C.c_double()
        _lib.check(L.atb_profile_read(k, _lib.C.byref(nl), _lib.C.byref(tm)))
        prof[name] = {"launches": nl.value, "ms": tm.value}
    # mass drift over the timed steps (reflective shell: mass is conserved)
    mj = torch.as_tensor(case.dg.MJ, device="cuda")
    m0, m1 = float((q0[0] * mj).sum()), float((q[0] * mj).sum())

    # e2e through the public API with host buffers (state in and out every step)
    qh = torch.empty(case.q0.shape, dtype=torch.float64, pin_memory=True)
    qh.copy_(torch.as_tensor(case.q0))
    qd = torch.empty_like(q)
    ke = max(3, min(steps, 20))
    qd.copy_(qh, non_blocking=True)
    s.step(qd, 1)
    qh.copy_(qd, non_blocking=True)
    barrier()
    e0.record(stream)
    for _ in range(ke):
        qd.copy_(qh, non_blocking=True)
        s.step(qd, 1)
        qh.copy_(qd, non_blocking=True)
    e1.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), dist)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    peak_fp64 = _lib.C.c_double()
    _lib.check(L.atb_probe_fp64_peak(_lib.C.byref(peak_fp64), _lib.stream_ptr()))
    peaks, kind = measured_peaks()

    def kern(name, flops_keys, label):
        t = prof[name]
        if not t["launches"]:
            return None
        avg = t["ms"] / t["launches"]
        fpd = sum(FLOPS_PER_DOF_STAGE[k] for k in flops_keys)
        fl = fpd * dofs
        return {"kernel": label, "avg_launch_ms": avg, "bound": "fp64", "flops_per_dof_stage": fpd,
                "achieved_tflops": fl / (avg * 1e-3) / 1e12,
                "peak_tflops": peak_fp64.value, "frac": fl / (avg * 1e-3) / 1e12 / peak_fp64.value}

    value = world * dofs * 3 * steps / (ms * 1e-3)
    # the stage kernel: the explicit EC tendency, fused with the radial linear
    # operator and the ARK accumulation when the solver fuses them
    fused = prof["tendency_linear"]["launches"] == 0
    tend = kern("tendency", ["sphere_N5_ec_rusanov"] + (["sphere_N5_linear_weak_z"] if fused else []),
                "curved_kernel<EulerGravity,EC,Rusanov,fused> (ARK23 stage: EC tendency + radial linear operator)"
                if fused else "curved_kernel<EulerGravity,EC> (explicit stage tendency)")
    lin = kern("tendency_linear", ["sphere_N5_linear_weak_z"],
               "curved_kernel<LinearEulerGravity,WEAK> (vertical linear operator + ARK accumulation)")
    b = prof["band_solve"]
    band = None
    if b["launches"]:
        avgb = b["ms"] / b["launches"]
        # per-line factors: every line reads its factor's nonzero structure
        # once -- per element block the dense diagonal block (L and U, BW1^2)
        # and the ns x ns face-coupling blocks of L below and U above it --
        # and the right-hand side, writes y, reads it back and writes x
        nlines = 6 * KH * KH * (N + 1) ** 2
        BW1 = 5 * (N + 1)
        byt = (nlines * (KV * BW1 * BW1 + 2 * (KV - 1) * 25) + 4 * dofs) * 8
        band = {"kernel": "band_solve_lines_kernel<6,5,sparse> (one factor per vertical line)", "avg_launch_ms": avgb,
                "bound": "hbm", "bytes_per_launch": byt, "achieved_gbs": byt / (avgb * 1e-3) / 1e9,
                "peak_gbs": peaks["hbm_gbs"], "frac": byt / (avgb * 1e-3) / 1e9 / peaks["hbm_gbs"],
                "peak_kind": kind}
    line = {
        "metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (the reference experiment's initial state)",
        "config": {"workload": f"3-D Euler-gravity acoustic wave on a cubed-sphere shell, 6x{KH}x{KH}x{KV} curved "
                               f"hexahedra, N={N} ({dofs} DOFs), EC volume + Rusanov surface flux, IMEX ARK23 "
                               "split_rhs=false, per-line vertical banded solve",
                   "dofs": dofs, "stages_per_step": 3, "dt_s": case.dt,
                   "l2": f"working set ~{dofs * 8 * 30 / 1e9:.1f} GB (state, stages, metrics, bands) > 126 MB L2"},
        "elements_per_cta": tuned, "gpu_launches": int(n1.value - n0.value),
        "setup_s": {"grid_and_initial_state_host": t_setup, "solver_with_band_factor": t_solver},
        "e2e": {"value": world * dofs * 3 * ke / (ms_e2e * 1e-3), "unit": "DOF-stage/s",
                "h2d_bytes_per_step": dofs * 8, "d2h_bytes_per_step": dofs * 8, "steps": ke},
        "roofline": tend and {"bound": "fp64", "kernel": tend["kernel"], "achieved": tend["achieved_tflops"],
                              "peak": tend["peak_tflops"], "unit": "TFLOP/s", "frac": tend["frac"],
                              "peak_source": "measured in this run: FP64 FMA probe (atb_probe_fp64_peak)",
                              "flops_per_dof_stage": tend["flops_per_dof_stage"], "traffic": None},
        "kernels": {"tendency": tend, "tendency_linear": lin, "band_solve": band, "launch_totals": prof},
        "mass_drift": abs(m1 - m0) / m0,
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as orc
        threads = os.cpu_count() or 1
        orc.set_threads(threads)
        qo = case.q0.copy()
        so = orc.ARK23(orc.DGSEM(case.dg), orc.DGSEM(case.lindg), qo, case.dt, split_rhs=False)
        so.step(qo, 1)
        n, T = _time_steps(so, qo, 10.0, 50)
        line["cpu_baseline"] = {"value": dofs * 3 * n / T, "unit": "DOF-stage/s", "cores": threads, "kind": "port",
                                "sample": f"{n} ARK23 steps of the same sphere workload, {threads} threads, "
                                          f"{T:.1f} s"}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ------------------------------------------- batched shallow-water instances
def run_swbatch(args):
    """256 rotating shallow-water instances (f-plane, g = 9.81), each a
    periodic 32 x 32 square of N = 4 elements with its own seeded bathymetry
    and height perturbation, packed into one operator (atb_op_create_batch)
    and stepped by LSRK54 with FP32 flux arithmetic and FP64 state.  Reports
    the packed FP32-flux throughput beside the packed FP64 run and the plain
    FP64 path (one instance at a time) on the same inputs, the relative L2
    error and mass drift against the FP64 run, and lake-at-rest residuals."""
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    dist, rank, world = dist_init()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    A = load_pkg()
    load_pkg()
    from atum_b200 import workloads as P

    n_inst, K, N = args.instances, 32, 4
    steps = args.steps if args.steps is not None else 500
    seeds = instance_seeds(n_inst, rank)

    def cases(precision, lake=False, n=n_inst):
        return [P.sw_fplane(N=N, K=K, seed=sd, precision=precision, lake_at_rest=lake, steps=steps)
                for sd in seeds[:n]]

    c32, c64 = cases("fp32flux"), cases("fp64")
    dt = min(c.dt for c in c64)
    p32 = A.batch.PackedDGSEM([c.dg for c in c32])
    p64 = A.batch.PackedDGSEM([c.dg for c in c64])
    q0 = p64.pack([torch.as_tensor(c.q0, device="cuda") for c in c64])
    dofs = q0.numel()
    MJ = torch.as_tensor(c64[0].dg.MJ, device="cuda")  # identical grids

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def timed(packed, q, nsteps, warm):
        s = A.LSRK54(packed, q, dt)
        s.step(q, warm)
        q.copy_(q0)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s.step(q, nsteps)
        e1.record()
        barrier()
        return e0.elapsed_time(e1)

    E32 = p32.autotune(q0.clone())
    E64 = p64.autotune(q0.clone())
    q32, q64 = q0.clone(), q0.clone()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms32 = timed(p32, q32, steps, args.warmup)
    ms64 = timed(p64, q64, steps, args.warmup)
    # persistent launches of the packed FP32-flux operator: k CTAs per SM walk
    # every instance's element tiles with a grid stride (same results)
    nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    persist = {}
    for k in (2, 4, 8, 16):
        qp = q0.clone()
        p32.set_persistent(nsm * k)
        msp = max_over_ranks(timed(p32, qp, steps, args.warmup), dist)
        persist[f"{k}_per_sm"] = {"ctas": nsm * k, "value": world * dofs * 5 * steps / (msp * 1e-3),
                                  "ms_per_step": msp / steps, "bitwise_equal_to_ordinary": bool(torch.equal(qp, q32))}
    p32.set_persistent(0)
    # plain FP64 path: the same instances one at a time (sample of 8)
    nseq = min(8, n_inst)
    qs = [torch.as_tensor(c.q0, device="cuda").contiguous() for c in c64[:nseq]]
    sol = [A.LSRK54(c.dg, q, dt) for c, q in zip(c64[:nseq], qs)]
    for s_, q in zip(sol, qs):
        s_.step(q, args.warmup)
    for c, q in zip(c64[:nseq], qs):
        q.copy_(torch.as_tensor(c.q0, device="cuda"))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for s_, q in zip(sol, qs):
        s_.step(q, steps)
    e1.record()
    barrier()
    ms_seq = e0.elapsed_time(e1)
    ms32, ms64, ms_seq = (max_over_ranks(x, dist) for x in (ms32, ms64, ms_seq))
    dofs_inst = dofs // n_inst

    # accuracy: per instance relative L2 (MJ-weighted) against the FP64 run
    def per_inst(q):
        return q.reshape(q.shape[0], n_inst, -1, q.shape[-1])

    a, b = per_inst(q32), per_inst(q64)
    w = MJ[None, None]
    err = torch.sqrt(((a - b) ** 2 * w).sum(dim=(0, 2, 3)) / (b ** 2 * w).sum(dim=(0, 2, 3)))
    mass0 = (per_inst(q0)[0] * MJ[None]).sum(dim=(1, 2))
    drift32 = ((a[0] * MJ[None]).sum(dim=(1, 2)) - mass0).abs() / mass0
    drift64 = ((b[0] * MJ[None]).sum(dim=(1, 2)) - mass0).abs() / mass0
    # lake at rest in the FP32-flux form: surface and velocity residuals
    nl = min(16, n_inst)
    cl = cases("fp32flux", lake=True, n=nl)
    pl = A.batch.PackedDGSEM([c.dg for c in cl])
    ql = pl.pack([torch.as_tensor(c.q0, device="cuda") for c in cl])
    bl = torch.cat([torch.as_tensor(c.dg.auxstate_host()[0], device="cuda") for c in cl], dim=0)
    A.LSRK54(pl, ql, dt).step(ql, steps)
    torch.cuda.synchronize()
    eta_res = float(((ql[0] + bl) - 100.0).abs().max())
    vel_res = float((ql[1:3].abs() / ql[0]).max())
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    total = world * dofs * 5 * steps
    v32 = total / (ms32 * 1e-3)
    v64 = total / (ms64 * 1e-3)
    vseq = dofs_inst * nseq * 5 * steps / (ms_seq * 1e-3)
    line = {
        "metric": "DOF-stage updates/s", "value": v32, "unit": "DOF-stage/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms32 / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64-state/f32-flux", "data": "synthetic",
        "config": {"workload": f"{n_inst} rotating shallow-water instances, periodic 32x32 elements, N=4, EC "
                               "volume + Rusanov surface flux, FP32 flux / FP64 state, LSRK54, one packed operator",
                   "instances": n_inst, "dofs": dofs, "stages_per_step": 5,
                   "l2": f"working set ~{3 * dofs * 8 / 1e9:.2f} GB > 126 MB L2 (no flush)",
                   "elements_per_cta": {"fp32flux": E32, "fp64": E64}},
        "packed_fp64": {"value": v64, "ms_per_step": ms64 / steps},
        "packed_fp32flux_persistent": persist,
        "plain_fp64_one_instance_at_a_time": {"value": vseq, "ms_per_step_per_instance": ms_seq / steps / nseq,
                                               "sample_instances": nseq},
        "speedup_vs_plain_fp64": v32 / vseq,
        "accuracy_vs_fp64": {"rel_l2_max": float(err.max()), "rel_l2_median": float(err.median()),
                             "mass_drift_max_fp32flux": float(drift32.max()),
                             "mass_drift_max_fp64": float(drift64.max())},
        "lake_at_rest_fp32flux": {"instances": nl, "max_abs_surface_residual_m": eta_res,
                                  "max_abs_velocity_m_per_s": vel_res},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def profiled_traffic(profile=PROFILE_TEND):
    """DRAM bytes (read + write) of one FP64 launch of the kernel and workload
    a committed ncu summary covers."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), profile)
    try:
        with open(path) as f:
            for ln in f:
                if ln.startswith("traffic_bytes_per_launch:"):
                    return int(ln.split(":")[1])
    except OSError:
        pass
    return None


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 100 for the bubble, 500 for the shallow-water batch)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32flux"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision-pair", action="store_true",
                    help="bubble: skip the FP32-flux run beside the FP64 headline")
    ap.add_argument("--elements-per-cta", type=int, default=0,
                    help="bubble: launch shape of the explicit operator (elements per CTA) instead of autotuning")
    ap.add_argument("--scheme", default="ark23", choices=sorted(SCHEME_STAGES),
                    help="time stepper of the bubble workload: IMEX ARK23 (default) or the fully explicit LSRK54 "
                         "run of the same problem")
    ap.add_argument("--workload", default="bubble", choices=["bubble", "swbatch", "serve", "c5", "sphere"],
                    help="bubble: 3-D rising bubble, IMEX ARK23 (default); swbatch: packed shallow-water "
                         "instances; serve: Poisson request stream through the serving loop; c5: 128x128x32 "
                         "hexahedra at N=7, FP64 and FP32-flux")
    ap.add_argument("--c5-elements", type=int, nargs=3, default=[128, 128, 32],
                    help="element counts of the c5 workload (smaller counts for a quick run)")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--time-scale", type=float, default=0.0005)
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    ap.add_argument("--pool-gb", type=float, default=12.0)
    ap.add_argument("--result-gb", type=float, default=16.0,
                    help="serve: page-locked host arena for result copies")
    ap.add_argument("--error-samples", type=int, default=16)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.workload == "swbatch":
        return run_swbatch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "sphere":
        return run_sphere(args)
    if args.workload == "c5":
        return run_c5(args)
    if args.steps is None:
        args.steps = 100
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
