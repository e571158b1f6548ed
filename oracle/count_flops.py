"""TEST INFRASTRUCTURE — algorithmic FP64 flop counts per DOF-stage from the
instrumented oracle (oracle.cpp's counting real type).

Recipe for the flux-differencing tendency (per element and stage):
  * every tensor line counts its UNORDERED node pairs once, Nq(Nq+1)/2, each
    costing one two-point flux as the reference evaluates it;
  * every ORDERED pair adds the reference's contraction 6*dim*Ns + 2*Ns
    (src/dgsem.jl:545-552) and, for Euler-gravity, the fluctuation term 3+dim;
  * every face node of every face adds one surface flux;
divided by Np*Ns DOFs.  + - * / count 1; sqrt and log count 1 and are also
reported separately.  Prints a JSON table used by bench.py.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "tests"))


def fd_flops(dg, vflux_kind, sflux_kind, q1, a1, q2, a2):
    import pyoracle as orc
    law = dg.law
    dim, Nq = law.dim, dg.grid.cell.Nq
    ns = law.numberofstates
    tp = orc.count_flops(dg, 1, vflux_kind, q1, a1, q2, a2, [0, 0, 1.0][:dim] + [0.0] * (3 - dim))
    sf = orc.count_flops(dg, 2, sflux_kind, q1, a1, q2, a2, [0, 0, 1.0][:dim] + [0.0] * (3 - dim))
    f_tp = sum(tp[k] for k in ("add", "mul", "div", "sqrt", "log", "pow"))
    f_sf = sum(sf[k] for k in ("add", "mul", "div", "sqrt", "log", "pow"))
    lines = dim * Nq ** (dim - 1)
    unordered = Nq * (Nq + 1) // 2
    ordered = Nq * Nq
    fluct = (3 + dim) if law.kind == 2 else 0
    per_elem = lines * (unordered * f_tp + ordered * (6 * dim * ns + 2 * ns + fluct))
    per_elem += 2 * dim * Nq ** (dim - 1) * f_sf
    dofs = Nq ** dim * ns
    logs = lines * unordered * tp["log"] / dofs
    return {"flops_per_dof_stage": per_elem / dofs, "logs_per_dof_stage": logs,
            "twopoint": tp, "surface": sf}


def weak_flops(dg, sflux_kind, q1, a1, q2, a2):
    """Weak-form operator restricted to its directions (the linear
    Euler-gravity operator of the IMEX stages, directions = (dim,)): per node
    the reference's full flux matrix, the D^T contraction of each active
    direction (Nq multiply-adds per state), the law's source (2 per
    dimension); per face node of each active direction's two faces one surface
    flux; divided by Np*Ns."""
    import pyoracle as orc
    law = dg.law
    dim, Nq = law.dim, dg.grid.cell.Nq
    ns = law.numberofstates
    nd = len(dg.directions)
    n = [0.0] * 3
    n[dg.directions[-1] - 1] = 1.0
    fx = orc.count_flops(dg, 0, 0, q1, a1, q2, a2, n)
    sf = orc.count_flops(dg, 2, sflux_kind, q1, a1, q2, a2, n)
    f_fx = sum(fx[k] for k in ("add", "mul", "div", "sqrt", "log", "pow"))
    f_sf = sum(sf[k] for k in ("add", "mul", "div", "sqrt", "log", "pow"))
    Np = Nq ** dim
    per_elem = Np * (f_fx + nd * 2 * Nq * ns + 2 * dim) + nd * 2 * Nq ** (dim - 1) * f_sf
    return {"flops_per_dof_stage": per_elem / (Np * ns), "flux": fx, "surface": sf}


def main():
    import problems as P
    out = {}
    case = P.bubble_3d(N=4, K=2, imex=True, steps=1)
    x = case.q0
    a = case.dg.auxstate_host()
    q1, q2, a1, a2 = x[:, 0, 0], x[:, 1, 7], a[:, 0, 0], a[:, 1, 7]
    out["bubble_3d_N4_ec_rusanov"] = fd_flops(case.dg, 2, 1, q1, a1, q2, a2)
    out["bubble_3d_N4_linear_weak_z"] = weak_flops(case.lindg, 1, q1, a1, q2, a2)
    c1 = P.vortex_c1()
    x = c1.q0
    out["vortex_2d_N3_ec_rusanov"] = fd_flops(c1.dg, 2, 1, x[:, 0, 0], [], x[:, 3, 5], [])
    c5 = P.bubble_3d(N=7, K=2, imex=True, steps=1)
    x = c5.q0
    a = c5.dg.auxstate_host()
    out["bubble_3d_N7_ec_rusanov"] = fd_flops(c5.dg, 2, 1, x[:, 0, 0], a[:, 0, 0], x[:, 1, 9], a[:, 1, 9])
    out["bubble_3d_N7_linear_weak_z"] = weak_flops(c5.lindg, 1, x[:, 0, 0], a[:, 0, 0], x[:, 1, 9], a[:, 1, 9])
    # cubed-sphere acoustic wave, N = 5 (the reference's contraction is the
    # curved-element one already: all three two-point flux rows with both
    # nodes' metric terms, so curvature changes no count)
    from atum_b200 import workloads as W
    sp = W.sphere_acoustic_wave(N=5, KH=1, KV=1, steps=1)
    x = sp.q0
    a = sp.dg.auxstate_host()
    out["sphere_N5_ec_rusanov"] = fd_flops(sp.dg, 2, 1, x[:, 0, 0], a[:, 0, 0], x[:, 1, 9], a[:, 1, 9])
    out["sphere_N5_linear_weak_z"] = weak_flops(sp.lindg, 1, x[:, 0, 0], a[:, 0, 0], x[:, 1, 9], a[:, 1, 9])
    print(json.dumps(out, indent=1, sort_keys=True))


if __name__ == "__main__":
    import importlib.util
    root = os.path.dirname(HERE)
    spec = importlib.util.spec_from_file_location("atum_b200", os.path.join(root, "atum.jl_b200", "__init__.py"),
                                                  submodule_search_locations=[os.path.join(root, "atum.jl_b200")])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["atum_b200"] = mod
    spec.loader.exec_module(mod)
    main()
