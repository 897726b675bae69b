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
    a = ap.parse_args()
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


if __name__ == "__main__":
    main()
