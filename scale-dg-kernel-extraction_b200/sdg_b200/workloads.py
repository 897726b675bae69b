"""Seeded synthetic workloads: the meshes, initial conditions, velocities and
instance compositions that the bench measures and the parity tests check.

The reference has no dataset; its runs are driven by input.conf (NeX, NeY,
NeZ, PolyOrder, dt, nstep).  Every workload here is a periodic unit box with
dt = 0.1 h / (p+1)^2, h = 1/max(NeX, NeY, NeZ), and the seeded initial
condition ic_kind = 1 (a Gaussian bump of sigma 0.1 at the centre plus eight
Fourier modes with integer wavenumbers 1..4 per axis and N(0, 0.01)
amplitudes).
"""
import numpy as np

# name: (NeX, NeY, NeZ, p, form, velocity, nstep)
#   form "GPU" = fast FP64, "OPT1"/"GENERAL" = bit-exact FP64 orders,
#   "MIXED" = FP32 state/derivatives with FP64 RK accumulation;
#   velocity: a constant (u, v, w) or "divfree" = (sin 2pi y, sin 2pi z,
#   sin 2pi x).
WORKLOADS = {
    "fp64_8c_p3": (8, 8, 8, 3, "GENERAL", (1.0, 0.5, 0.25), 100),
    "fp64_32c_p7": (32, 32, 32, 7, "GPU", (1.0, 0.5, 0.25), 200),
    "mixed_32c_p7": (32, 32, 32, 7, "MIXED", "divfree", 200),
    "mixed_16c_p15": (16, 16, 16, 15, "MIXED", "divfree", 200),
}

IC_SEED = 2024


def dt_for(ne_max, p):
    return 0.1 / ne_max / (p + 1) ** 2


def fields_kwargs(vel):
    """init_fields keyword arguments for a workload's velocity entry."""
    if vel == "divfree":
        return {"ic_kind": 1, "seed": IC_SEED, "vel_kind": 1}
    return {"ic_kind": 1, "seed": IC_SEED, "vel_kind": 0, "vel": tuple(vel)}


def ensemble_instances(n, seed, ne_range, p_choices, rng_nstep=None):
    """Seeded instance list: cubic boxes Ne ~ U{ne_range} per axis, p from
    p_choices, constant velocity U[-1,1]^3 (drawn from the instance seed),
    dt = 0.1 h / (p+1)^2, and optionally nstep ~ U{rng_nstep}."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        ne = int(rng.integers(ne_range[0], ne_range[1] + 1))
        p = int(rng.choice(p_choices))
        nstep = int(rng.integers(rng_nstep[0], rng_nstep[1] + 1)) if rng_nstep else None
        out.append({"ne": ne, "p": p, "seed": 1000 + k, "nstep": nstep,
                    "dt": dt_for(ne, p)})
    return out


def batch_composition():
    """The batched ensemble: 96 instances, Ne per axis U{6..24}, p in
    {3, 5, 7, 9}; 100 steps each."""
    return ensemble_instances(96, 4, (6, 24), [3, 5, 7, 9])


def served_stream(nreq):
    """The served request stream: Ne per axis U{8..32}, p U{3..11}, nstep
    U{50..400}, and an FP32/FP64 flag per request."""
    reqs = ensemble_instances(nreq, 5, (8, 32), list(range(3, 12)), (50, 400))
    rng = np.random.default_rng(6)
    for r in reqs:
        r["mixed"] = bool(rng.integers(0, 2))
    return reqs, rng
