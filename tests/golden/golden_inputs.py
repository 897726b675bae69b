"""Cases and seeded inputs of the golden fixtures (shared by make_golden.py
and the tests).  Inputs come from splitmix64 integer arithmetic, so every
machine regenerates them bit for bit."""
import numpy as np

MESH_CASES = [(2, 3, 2, 1), (3, 2, 2, 2), (2, 2, 3, 3), (1, 2, 1, 7)]

# (evaluation type, p, (NeX, NeY, NeZ))
TEND_CASES = [
    ("GENERAL", 1, (2, 2, 2)), ("OPT1", 1, (2, 2, 2)),
    ("GENERAL", 2, (2, 1, 2)), ("OPT1", 3, (2, 2, 1)),
    ("GENERAL", 4, (1, 2, 2)), ("OPT1", 5, (1, 1, 2)),
    ("OPT1", 7, (2, 1, 1)), ("GENERAL", 7, (1, 1, 1)),
    ("OPT1", 8, (1, 1, 1)), ("GENERAL", 8, (1, 1, 1)),
    ("OPT1", 11, (1, 1, 1)), ("GENERAL", 11, (1, 1, 1)),
    ("OPT1", 15, (1, 1, 1)), ("GENERAL", 15, (1, 1, 1)),
]

MAIN_CASES = {
    "opt1_p3": """&PARAM_ADVECT3D
  NeX = 2,
  NeY = 2,
  NeZ = 2,
  PolyOrder = 3,
  DGOptrKernel_OptType = "OPT1" ! GENERAL or OPT1
  dt    = 2.0D-3,
  nstep = 12,
  output_interval = 4,
/
""",
    "general_p2_vel": """&PARAM_ADVECT3D
  NeX = 3, NeY = 2, NeZ = 2,
  PolyOrder = 2,
  vel_x = 1.0, vel_y = -0.5, vel_z = 0.25,
  DGOptrKernel_OptType = "GENERAL"
  dt = 1.0D-3, nstep = 6, output_interval = 3,
/
""",
    "opt1_p9": """&PARAM_ADVECT3D
  NeX = 1, NeY = 1, NeZ = 2,
  PolyOrder = 9,
  DGOptrKernel_OptType = "OPT1"
  dt = 2.0D-4, nstep = 2, output_interval = 1,
/
""",
}

_C0 = np.uint64(0x9E3779B97F4A7C15)
_C1 = np.uint64(0xBF58476D1CE4E5B9)
_C2 = np.uint64(0x94D049BB133111EB)


def splitmix_uniform(seed, n):
    """n doubles in [0,1) from the splitmix64 stream of `seed`."""
    with np.errstate(over="ignore"):
        s = np.uint64(seed) + np.arange(1, n + 1, dtype=np.uint64) * _C0
        z = (s ^ (s >> np.uint64(30))) * _C1
        z = (z ^ (z >> np.uint64(27))) * _C2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def tend_inputs(p, dims, Np, NeA):
    """q in [-1,1), u,v,w in [-1,1) plus an offset, shape (Np, NeA); the
    halo part is overwritten by update_halo before use."""
    seed = 1000 * p + 100 * dims[0] + 10 * dims[1] + dims[2]
    n = Np * NeA
    out = []
    for k, off in enumerate((0.0, 0.3, -0.2, 0.1)):
        x = 2.0 * splitmix_uniform(seed + 7919 * k, n) - 1.0 + off
        out.append(x.reshape(Np, NeA, order="F"))
    return out
