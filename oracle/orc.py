"""ctypes binding of the CPU oracle (liboracle_sdg.so).

TEST INFRASTRUCTURE ONLY: the test-suite, the smoke check and the bench's
CPU-baseline leg use it as the checker.  The product never imports it.

The oracle restates the reference Fortran loop for loop (see sdg_oracle.h);
arrays use the reference's Fortran layout (numpy order="F", 1-based maps).
"""

import ctypes
import os
import subprocess
from collections import namedtuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_sdg.so")
CLI_PATH = os.path.join(HERE, "sdg_oracle")
OPERATOR_DIR = os.path.join(os.path.dirname(HERE), "operator_data")

GENERAL = 1
OPT1 = 2

_I, _D, _P, _U64 = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_ulonglong
_SIGS = {
    "orc_read_operators": (_I, [ctypes.c_char_p, _I, _P, _P, _P]),
    "orc_mesh_sizes": (_I, [_I, _I, _I, _I, _P]),
    "orc_fmask": (None, [_I, _P]),
    "orc_mesh_setup": (_I, [_I, _I, _I, _I, _D, _D, _D, _P, _P, _P, _P, _P, _P, _P, _P]),
    "orc_update_halo": (None, [_P, _I, _I, _I, _P]),
    "orc_cal_tend": (_I, [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                          _I, _I, _I, _I, _I, _P, _P]),
    "orc_run_rk3": (_I, [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                         _I, _I, _I, _I, _D, _I, _I, _P, _P]),
    "orc_init_fields": (_I, [_I, _U64, _I, _D, _D, _D, _P, _I, _I, _I, _P, _P, _P, _P]),
    "orc_random_velocity": (None, [_U64, _P]),
    "orc_num_threads": (_I, []),
    "orc_divlike_fields": (_I, [_I, _I, _I, ctypes.c_longlong, _P, _P, _P, _P, _P, _P, _P]),
}

_lib = None


def build():
    """Compiles the oracle with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


Ops = namedtuple("Ops", "p Nq x1D D1D D1D_tr Lift_mat")
Mesh = namedtuple(
    "Mesh",
    "NeX NeY NeZ p Nq Np NfpTot Ne Nhalo NeA NhaloNode "
    "VMapM VMapP halo_src_map normal_fn Escale Fscale pos_en",
)


def read_operators(p, opdir=OPERATOR_DIR):
    Nq = p + 1
    x = np.zeros(Nq)
    D = np.zeros((Nq, Nq), order="F")
    L = np.zeros((Nq, Nq, Nq, 6), order="F")
    rc = lib().orc_read_operators(opdir.encode(), p, _p(x), _p(D), _p(L))
    if rc:
        raise IOError(f"oracle: cannot read operators p={p} ({rc})")
    return Ops(p, Nq, x, D, np.asfortranarray(D.T), L)


def fmask(p):
    Nq = p + 1
    F = np.zeros((Nq * Nq, 6), dtype=np.int32, order="F")
    lib().orc_fmask(Nq, _p(F))
    return F


def mesh_setup(NeX, NeY, NeZ, p, x1D, dom=(1.0, 1.0, 1.0)):
    s = np.zeros(6, dtype=np.int32)
    lib().orc_mesh_sizes(NeX, NeY, NeZ, p, _p(s))
    Ne, Nhalo, NeA, NhaloNode, Np, NfpTot = map(int, s)
    VMapM = np.zeros((NfpTot, Ne), dtype=np.int32, order="F")
    VMapP = np.zeros((NfpTot, Ne), dtype=np.int32, order="F")
    hmap = np.zeros(NhaloNode, dtype=np.int32)
    nfn = np.zeros((NfpTot, Ne, 3), order="F")
    Esc = np.zeros((Np, Ne, 3), order="F")
    Fsc = np.zeros((NfpTot, Ne), order="F")
    pos = np.zeros((Np, Ne, 3), order="F")
    x1D = np.ascontiguousarray(x1D, dtype=np.float64)
    lib().orc_mesh_setup(NeX, NeY, NeZ, p, dom[0], dom[1], dom[2], _p(x1D), _p(VMapM),
                         _p(VMapP), _p(hmap), _p(nfn), _p(Esc), _p(Fsc), _p(pos))
    return Mesh(NeX, NeY, NeZ, p, p + 1, Np, NfpTot, Ne, Nhalo, NeA, NhaloNode, VMapM,
                VMapP, hmap, nfn, Esc, Fsc, pos)


def update_halo(f, mesh):
    lib().orc_update_halo(_p(f), mesh.Np, mesh.Ne, mesh.NhaloNode, _p(mesh.halo_src_map))
    return f


def init_fields(mesh, ic_kind=0, seed=0, vel_kind=0, vel=(1.0, 1.0, 1.0)):
    shape = (mesh.Np, mesh.NeA)
    q, u, v, w = (np.zeros(shape, order="F") for _ in range(4))
    rc = lib().orc_init_fields(ic_kind, seed, vel_kind, vel[0], vel[1], vel[2],
                               _p(mesh.pos_en), mesh.Np, mesh.Ne, mesh.NeA, _p(q), _p(u),
                               _p(v), _p(w))
    if rc:
        raise ValueError(f"oracle: bad init kind ({rc})")
    for f in (q, u, v, w):
        update_halo(f, mesh)
    return q, u, v, w


def random_velocity(seed):
    out = np.zeros(3)
    lib().orc_random_velocity(seed, _p(out))
    return out


def cal_tend(evaltype, q, u, v, w, ops, mesh, times=None):
    """advect3d_eq_cal_tend restated; returns dqdt (Np,NeA), halo part 0."""
    m = mesh
    dqdt = np.zeros((m.Np, m.NeA), order="F")
    tf, td = ctypes.c_double(0.0), ctypes.c_double(0.0)
    rc = lib().orc_cal_tend(evaltype, _p(dqdt), _p(q), _p(u), _p(v), _p(w), _p(ops.D1D),
                            _p(ops.D1D_tr), _p(ops.Lift_mat), _p(m.VMapM), _p(m.VMapP),
                            _p(m.normal_fn), _p(m.Escale), _p(m.Fscale), m.Nq, m.Np,
                            m.NfpTot, m.Ne, m.NeA, ctypes.byref(tf), ctypes.byref(td))
    if rc:
        raise ValueError(f"oracle: cal_tend failed ({rc})")
    if times is not None:
        times.extend([tf.value, td.value])
    return dqdt


def run_rk3(evaltype, q, u, v, w, ops, mesh, dt, nstep, output_interval=0):
    """SSP-RK3 loop of main.f90:51-80 on q (updated in place).

    Returns (diag, times): diag rows (istep, min, max); times = Main,
    Cal_tend, flux, dqdt seconds."""
    m = mesh
    nd = nstep // output_interval if output_interval > 0 else 0
    diag = np.zeros(3 * max(nd, 1))
    times = np.zeros(4)
    rc = lib().orc_run_rk3(evaltype, _p(q), _p(u), _p(v), _p(w), _p(ops.D1D),
                           _p(ops.Lift_mat), _p(m.VMapM), _p(m.VMapP),
                           _p(m.halo_src_map), _p(m.normal_fn), _p(m.Escale),
                           _p(m.Fscale), m.Nq, m.Ne, m.NeA, m.NhaloNode, dt, nstep,
                           output_interval, _p(diag), _p(times))
    if rc:
        raise ValueError(f"oracle: run_rk3 failed ({rc})")
    return diag[: 3 * nd].reshape(nd, 3) if nd else np.zeros((0, 3)), times


def num_threads():
    return int(lib().orc_num_threads())


def divlike_fields(evaltype, D1D, nvar, Ne, ix, iy, iz):
    """divlike_dirXYZ_var5 / gradlike_dirXYZ restated (sdg_oracle.h): arrays of
    Ne*nvar*Np values, unit (element e, field v) at Np*(v + nvar*e); returns
    (ox, oy, oz)."""
    D = np.asarray(D1D, dtype=np.float64, order="F")
    Nq = D.shape[0]
    ix, iy, iz = (np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (ix, iy, iz))
    outs = [np.empty_like(ix) for _ in range(3)]
    rc = lib().orc_divlike_fields(evaltype, Nq, nvar, Ne, _p(D), _p(ix), _p(iy), _p(iz),
                                  *[_p(o) for o in outs])
    if rc:
        raise ValueError(f"oracle: divlike_fields failed ({rc})")
    return tuple(outs)
