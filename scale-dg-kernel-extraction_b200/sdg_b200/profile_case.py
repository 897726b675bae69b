"""A short, bounded run of the fused stage kernels for profilers.

Sets up one mesh, uploads the seeded state, runs `--warm` RK3 steps and then
`--launches` single stage launches (stages 1, 2, 3 in turn), and exits.
Meant to be wrapped by a profiler capturing a handful of launches, e.g.

  ncu --set full --clock-control none -k regex:tend_kernel -s 6 -c 3 \\
      python -m sdg_b200.profile_case --mesh 32 --p 7

(run from the package directory, or with it on PYTHONPATH).
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import sdg_b200 as sdg  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", type=int, default=32, help="elements per axis")
    ap.add_argument("--p", type=int, default=7)
    ap.add_argument("--mode", default="GPU", choices=["GPU", "OPT1", "GENERAL", "MIXED"])
    ap.add_argument("--warm", type=int, default=2, help="RK3 steps before the launches")
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--op", default="stage", choices=["stage", "divlike"],
                    help="stage: fused RK stage kernels; divlike: the five-field "
                         "derivative operator (sdg_divlike_dev) on the same mesh")
    a = ap.parse_args()
    if a.op == "divlike":
        return divlike_case(a)
    flags = {"GPU": 0, "OPT1": sdg.FLAG_EXACT,
             "GENERAL": sdg.FLAG_EXACT | sdg.FLAG_ORDER_GENERAL,
             "MIXED": sdg.FLAG_MIXED}[a.mode]
    ops = sdg.read_operators(a.p)
    mesh = sdg.mesh_setup(a.mesh, a.mesh, a.mesh, a.p, ops.x1D)
    vel_kind = 1 if a.mode == "MIXED" else 0
    q, u, v, w = sdg.init_fields(mesh, ic_kind=1, seed=2024, vel_kind=vel_kind,
                                 vel=(1.0, 0.5, 0.25))
    h = sdg.Handle(ops, mesh, flags)
    h.set_state(q, u, v, w)
    dt = 0.1 / a.mesh / (a.p + 1) ** 2
    h.rk3_steps(dt, a.warm)
    for i in range(a.launches):
        h.rk3_stage(1 + i % 3, dt)
    h.synchronize()
    mn, mx = h.minmax()
    h.close()
    print(f"profile_case done: {a.mesh}^3 p={a.p} {a.mode}, min {mn:.6e} max {mx:.6e}")


def divlike_case(a):
    """--warm + --launches calls of sdg_divlike_dev (five seeded fields per
    element of a mesh^3 box at order p, FMA form)."""
    import torch
    nvar = 5
    ops = sdg.read_operators(a.p)
    Ne = a.mesh ** 3
    n = Ne * nvar * (a.p + 1) ** 3
    gen = torch.Generator(device="cuda").manual_seed(7)
    ins = [torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) for _ in range(3)]
    outs = [torch.empty_like(ins[0]) for _ in range(3)]
    for _ in range(a.warm + a.launches):
        sdg.divlike_dirXYZ_var_dev(ops.D1D, nvar, Ne, *ins, *outs)
    torch.cuda.synchronize()
    print(f"profile_case done: divlike {a.mesh}^3 p={a.p} x{nvar}, "
          f"|out_x| max {float(outs[0].abs().max()):.6e}")


if __name__ == "__main__":
    main()
