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
sys.path.insert(0, os.path.join(ROOT, "tests"))

# Algorithmic FP64 flops per DOF-stage of the flux-differencing tendency
# (EC volume flux, Rusanov surface flux), from the oracle's instrumented
# counter: python oracle/count_flops.py
FLOPS_PER_DOF_STAGE = {"bubble_3d_N4_ec_rusanov": 602.8, "bubble_3d_N7_ec_rusanov": 896.2}
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


def build_case(precision="fp64", K=16):
    import problems as P
    return P.bubble_3d(N=4, K=K, imex=True, steps=200, precision=precision)


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        return dist, int(os.environ.get("RANK", "0")), world
    return None, 0, 1


# ----------------------------------------------------------- reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as orc
    load_pkg()
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    case = build_case_sample()
    dg = orc.DGSEM(case.dg)
    lin = orc.DGSEM(case.lindg)
    q = case.q0.copy()
    s = orc.ARK23(dg, lin, q, case.dt, split_rhs=False)
    dofs = q.size
    s.step(q, args.warmup)
    t0 = time.perf_counter()
    s.step(q, args.steps)
    T = time.perf_counter() - t0
    v = dofs * 3 * args.steps / T
    sample = (f"{case.dg.grid.Kd[0]}x{case.dg.grid.Kd[1]}x{case.dg.grid.Kd[2]} elements (a horizontal "
              f"sub-sample of the 16x16x16 workload, same columns), {dofs} DOFs, ARK23 steps")
    line = {"metric": "DOF-stage updates/s", "value": v, "unit": "DOF-stage/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": T / args.steps * 1e3, "higher_is_better": True,
            "impl": "reference", "dtype": "f64", "data": "synthetic",
            "config": {"workload": "3-D Euler-gravity rising bubble, 16^3 hexahedra, N=4, FP64, IMEX ARK23 "
                                   "(CPU: horizontal sub-sample)", "sample": sample},
            "cpu_baseline": {"value": v, "unit": "DOF-stage/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "vs_baseline": None}
    print(json.dumps(line), flush=True)
    return 0


def build_case_sample():
    """Horizontal sub-sample of the benchmark workload: 4x4 of the 16x16
    element columns at full height, identical spacing, physics and dt."""
    import numpy as np
    import problems as P
    import atum_b200 as A
    full = build_case()
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
    return P.Case("bubble_3d_sample", dg, q0, full.dt, full.timeend, solver="ARK23", lindg=lin, split_rhs=False,
                  adjust_final=False)


def cpu_baseline_sample():
    """Oracle port on the host cores: one ARK23 step of the horizontal sub-sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as orc
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    case = build_case_sample()
    dg = orc.DGSEM(case.dg)
    lin = orc.DGSEM(case.lindg)
    q = case.q0.copy()
    s = orc.ARK23(dg, lin, q, case.dt, split_rhs=False)
    s.step(q, 1)
    n = 2
    t0 = time.perf_counter()
    s.step(q, n)
    T = time.perf_counter() - t0
    return {"value": q.size * 3 * n / T, "unit": "DOF-stage/s", "cores": threads, "kind": "port",
            "sample": f"{n} ARK23 steps of a 4x4x16-element horizontal sub-sample ({q.size} DOFs) of the same "
                      f"workload, {threads} threads"}


# ---------------------------------------------------------------- our arm
def run_ours(args):
    import numpy as np
    import torch

    dist, rank, world = dist_init()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    A = load_pkg()
    from atum_b200 import _lib

    case = build_case(args.precision)
    dofs = case.q0.size
    q = torch.as_tensor(case.q0, device="cuda").contiguous()
    solver = A.ARK23(case.dg, case.lindg, q, case.dt, split_rhs=False)
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
    _lib.check(L.atb_profile_reset())
    _lib.check(L.atb_profile_enable(1))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        barrier()
        ev0.record(stream)
        solver.step(q, args.steps)
        ev1.record(stream)
        barrier()
    _lib.check(L.atb_profile_enable(0))
    ms = ev0.elapsed_time(ev1)
    n1 = _lib.C.c_long()
    L.atb_launch_count(_lib.C.byref(n1))
    prof = {}
    for k, name in enumerate(("tendency", "tendency_linear", "band_solve", "combine", "reduce")):
        nl, tm = _lib.C.c_long(), _lib.C.c_double()
        _lib.check(L.atb_profile_read(k, _lib.C.byref(nl), _lib.C.byref(tm)))
        prof[name] = {"launches": nl.value, "ms": tm.value}
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    assert torch.isfinite(q).all(), "non-finite state after the timed steps"

    # ------------------------------------------------------------- e2e
    # Through the public API with host buffers: every step copies the state
    # from pinned host memory to the device and the result back.
    qh = torch.empty(case.q0.shape, dtype=torch.float64, pin_memory=True)
    qh.copy_(torch.as_tensor(case.q0))
    qd = torch.empty_like(q)
    s2 = A.ARK23(case.dg, case.lindg, qd, case.dt, split_rhs=False)
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
    if dist is not None:
        t = torch.tensor([ms_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    value = world * dofs * 3 * args.steps / (ms * 1e-3)
    e2e = world * dofs * 3 * ke / (ms_e2e * 1e-3)
    tend = prof["tendency"]
    avg_ms = tend["ms"] / max(1, tend["launches"])
    key = "bubble_3d_N4_ec_rusanov"
    flops_launch = FLOPS_PER_DOF_STAGE[key] * dofs
    tflops = flops_launch / (avg_ms * 1e-3) / 1e12
    peak_fp64 = _lib.C.c_double()
    _lib.check(L.atb_probe_fp64_peak(_lib.C.byref(peak_fp64), _lib.stream_ptr()))
    peaks, kind = measured_peaks()
    # algorithmic bytes of the fused FP64 tendency launch: q (5 values) read,
    # ex_K (5) written, Phi (1) read = 11 x 8 B per node
    bytes_launch = 11 * 8 * dofs // 5
    line = {
        "metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64-state/f32-flux",
        "data": "synthetic",
        "config": {"workload": "3-D Euler-gravity rising bubble, 16^3 hexahedra, N=4 (2,560,000 DOFs), EC volume + "
                               "Rusanov surface flux, IMEX ARK23 split_rhs=false, vertical banded solve",
                   "dofs": dofs, "stages_per_step": 3, "precision": args.precision,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "working set ~0.21 GB > 126 MB L2 (no flush)"},
        "e2e": {"value": e2e, "unit": "DOF-stage/s", "h2d_bytes_per_step": dofs * 8, "d2h_bytes_per_step": dofs * 8,
                "steps": ke},
        "gpu_launches": int(n1.value - n0.value),
        "roofline": {"bound": "fp64", "kernel": "tendency_kernel<EulerGravity,3,EC> (nonlinear stage tendency)",
                     "achieved": tflops, "peak": peak_fp64.value, "unit": "TFLOP/s",
                     "frac": tflops / peak_fp64.value if peak_fp64.value > 0 else None,
                     "peak_source": "measured in this run: FP64 FMA probe (atb_probe_fp64_peak)",
                     "flops_per_launch": flops_launch, "avg_launch_ms": avg_ms,
                     "traffic": profiled_traffic() if args.precision == "fp64" else None,
                     "traffic_unit": "bytes per launch (dram read + write, one ncu capture)",
                     "traffic_source": PROFILE_TEND,
                     "hbm_view": {"bytes_per_launch": bytes_launch,
                                  "achieved_gbs": bytes_launch / (avg_ms * 1e-3) / 1e9,
                                  "peak_gbs": peaks["hbm_gbs"], "peak_kind": kind}},
        "kernels": prof,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample()
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


PROFILE_TEND = "profiles/tendency_eg3_ec_nq5_bubble16.md"


def profiled_traffic():
    """DRAM bytes (read + write) of one FP64 tendency launch of this workload,
    from the committed ncu summary of the same kernel and workload."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), PROFILE_TEND)
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
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32flux"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
