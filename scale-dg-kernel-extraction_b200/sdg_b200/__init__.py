"""Python binding of the B200 SCALE-DG advection library (libsdg_gpu.so).

A thin ctypes layer over the C ABI declared in include/sdg_gpu.h.  Arrays
use the reference's Fortran layout: numpy arrays in column-major order
(``order="F"``) with the reference's shapes, e.g. ``q`` is ``(Np, NeA)``,
``VMapM`` is ``(NfpTot, Ne)`` and holds 1-based indices.

The module mirrors the reference's driver surface:

* ``dg_optr_kernel_setup(evaltype)`` - the selector of
  mod_dg_optr_kernel.f90:45-58; "GPU" picks the fast FMA kernels, "OPT1" and
  "GENERAL" reproduce those CPU kernels' rounding bit for bit on the GPU;
* ``advect3d_eq_cal_tend(dqdt, q, u, v, w, D1D, D1D_tr, Lift_mat, VMapM,
  VMapP, normal_fn, Escale, Fscale, Nq, Np, NfpTot, Ne, NeA)`` - the
  tendency call of mod_advect3d_eq.f90:41-85 with the same arguments;
* ``mesh_setup`` / ``read_operators`` / ``update_halo`` - mod_mesh.f90.

There is no CPU path: every compute call runs the CUDA library, and a
missing library or device raises ``SdgError``.
"""

import ctypes
import os
from collections import namedtuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.dirname(_HERE)
REPO_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(PKG_DIR, "libsdg_gpu.so")
OPERATOR_DIR = os.path.join(REPO_DIR, "operator_data")

SDG_OK = 0
SDG_ERR_ARG = 1
SDG_ERR_CUDA = 2
SDG_ERR_IO = 3
SDG_ERR_MESH = 4
SDG_ERR_STATE = 5

FLAG_EXACT = 1
FLAG_ORDER_GENERAL = 2
FLAG_MIXED = 4
FLAG_EXTERNAL_HALO = 8

FIELD_Q, FIELD_U, FIELD_V, FIELD_W = 0, 1, 2, 3
ARRAY_STAGE2, ARRAY_STAGE3 = 4, 5

VARIANT_AUTO, VARIANT_BLOCK, VARIANT_PIPE, VARIANT_BLOCK8, VARIANT_SPLIT = 0, 1, 2, 3, 4
VARIANT_TENSOR = 5

# Exported symbols and their signatures (must match include/sdg_gpu.h).
_I, _D, _P, _LL = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong
_U64 = ctypes.c_ulonglong
SIGNATURES = {
    "sdg_last_error": (_I, [ctypes.c_char_p, _I]),
    "sdg_version": (ctypes.c_char_p, []),
    "sdg_read_operators": (_I, [ctypes.c_char_p, _I, _P, _P, _P]),
    "sdg_mesh_sizes": (_I, [_I, _I, _I, _I, _P]),
    "sdg_fmask": (_I, [_I, _P]),
    "sdg_mesh_setup": (_I, [_I, _I, _I, _I, _D, _D, _D, _P, _P, _P, _P, _P, _P, _P, _P]),
    "sdg_update_halo_host": (_I, [_P, _I, _I, _I, _P]),
    "sdg_init_fields": (_I, [_I, _U64, _I, _D, _D, _D, _P, _I, _I, _P, _P, _P, _P]),
    "sdg_random_velocity": (_I, [_U64, _P]),
    "sdg_box_fields": (_I, [_I, _I, _I, _I, _P, _I, _U64, _I, _D, _D, _D, _P, _P, _P, _P]),
    "sdg_init": (_I, [ctypes.POINTER(_P), _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P,
                      _P, _P, _P, _I]),
    "sdg_finalize": (_I, [_P]),
    "sdg_cal_tend": (_I, [_P, _P, _P, _P, _P, _P]),
    "sdg_cal_tend_dev": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "sdg_update_halo_dev": (_I, [_P, _P, _P]),
    "sdg_set_field": (_I, [_P, _I, _P]),
    "sdg_get_field": (_I, [_P, _I, _P]),
    "sdg_rk3_steps": (_I, [_P, _D, _I]),
    "sdg_rk3_steps_host": (_I, [_P, _P, _D, _I]),
    "sdg_minmax": (_I, [_P, _P, _P]),
    "sdg_diagnostics": (_I, [_P, _P, _D, _P, _P]),
    "sdg_synchronize": (_I, [_P]),
    "sdg_rk3_stage": (_I, [_P, _I, _D]),
    "sdg_get_stream": (_I, [_P, ctypes.POINTER(_P)]),
    "sdg_field_dev_ptr": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "sdg_timers": (_I, [_P, _P]),
    "sdg_resident_array": (_I, [_P, _I, ctypes.POINTER(_P), ctypes.POINTER(_I)]),
    "sdg_update_halo_stage": (_I, [_P, _I]),
    "sdg_launch_count": (_LL, [_P]),
    "sdg_set_kernel_variant": (_I, [_P, _I]),
    "sdg_debug_inject_wait_timeout": (_I, [_P, _I, _I]),
    "sdg_debug_chunk_bounds": (_I, [_I, _I, _I, _P, _I, ctypes.POINTER(_I)]),
    "sdg_debug_step_plan": (_I, [_I, _P, _P, _I, _I, _P, _I, ctypes.POINTER(_I)]),
    "sdg_minmax_dev_noalloc": (_I, [_P, _LL, _P, _P]),
    "sdg_divlike_dev": (_I, [_I, _I, _LL, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "sdg_gradlike_dev": (_I, [_I, _LL, _P, _P, _P, _P, _P, _I, _P]),
    "sdg_batch_create": (_I, [ctypes.POINTER(_P), _I]),
    "sdg_batch_add": (_I, [_P, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _D,
                           ctypes.POINTER(_I)]),
    "sdg_batch_commit": (_I, [_P, _I]),
    "sdg_batch_run": (_I, [_P, _I]),
    "sdg_batch_get": (_I, [_P, _I, _P]),
    "sdg_batch_info": (_I, [_P, _P, _I]),
    "sdg_batch_destroy": (_I, [_P]),
    "sdg_batch_debug_inject_wait_timeout": (_I, [_P, _I, _I]),
    "sdg_serve_create": (_I, [ctypes.POINTER(_P), _D]),
    "sdg_serve_submit": (_I, [_P, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _D, _I, _I,
                              ctypes.POINTER(_I)]),
    "sdg_serve_poll": (_I, [_P, _I, ctypes.POINTER(_I), _P]),
    "sdg_serve_result": (_I, [_P, _I, _P]),
    "sdg_serve_wait": (_I, [_P, _D]),
    "sdg_serve_stats": (_I, [_P, _P]),
    "sdg_serve_destroy": (_I, [_P]),
}


class SdgError(RuntimeError):
    """A failed library call; ``code`` is the SDG_ERR_* status."""

    def __init__(self, code, msg):
        super().__init__(f"[sdg status {code}] {msg}")
        self.code = code


_lib = None


def lib():
    """Loads libsdg_gpu.so once; raises SdgError when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SdgError(SDG_ERR_CUDA, f"{LIB_PATH} is not built (run build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != SDG_OK:
        buf = ctypes.create_string_buffer(1024)
        lib().sdg_last_error(buf, 1024)
        raise SdgError(rc, buf.value.decode(errors="replace"))


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _f64(a, shape=None):
    a = np.asarray(a, dtype=np.float64, order="F")
    if shape is not None and a.size != int(np.prod(shape)):
        raise SdgError(SDG_ERR_ARG, f"array of {a.size} values where {shape} expected")
    return a


def _i32(a):
    return np.asarray(a, dtype=np.int32, order="F")


# ---------------------------------------------------------------------------
# Host set-up (mod_mesh.f90)
# ---------------------------------------------------------------------------
Operators = namedtuple("Operators", "p Nq x1D D1D D1D_tr Lift_mat")
Mesh = namedtuple(
    "Mesh",
    "NeX NeY NeZ p Nq Np Nfp NfpTot Ne Nhalo NeA NhaloNode "
    "VMapM VMapP halo_src_map normal_fn Escale Fscale pos_en",
)


def read_operators(p, opdir=OPERATOR_DIR):
    """element_init operator read (mod_mesh.f90:253-263)."""
    Nq = p + 1
    x1D = np.zeros(Nq)
    D1D = np.zeros((Nq, Nq), order="F")
    Lift = np.zeros((Nq, Nq, Nq, 6), order="F")
    _check(lib().sdg_read_operators(opdir.encode(), p, _p(x1D), _p(D1D), _p(Lift)))
    return Operators(p, Nq, x1D, D1D, np.asfortranarray(D1D.T), Lift)


def mesh_sizes(NeX, NeY, NeZ, p):
    s = np.zeros(6, dtype=np.int32)
    _check(lib().sdg_mesh_sizes(NeX, NeY, NeZ, p, _p(s)))
    return dict(zip(["Ne", "Nhalo", "NeA", "NhaloNode", "Np", "NfpTot"], map(int, s)))


def fmask(p):
    Nq = p + 1
    F = np.zeros((Nq * Nq, 6), dtype=np.int32, order="F")
    _check(lib().sdg_fmask(p, _p(F)))
    return F


def mesh_setup(NeX, NeY, NeZ, p, x1D, dom=(1.0, 1.0, 1.0)):
    """mesh_setup (mod_mesh.f90:74-193): all tables, reference layout."""
    s = mesh_sizes(NeX, NeY, NeZ, p)
    Ne, NfpTot, Np = s["Ne"], s["NfpTot"], s["Np"]
    VMapM = np.zeros((NfpTot, Ne), dtype=np.int32, order="F")
    VMapP = np.zeros((NfpTot, Ne), dtype=np.int32, order="F")
    hmap = np.zeros(s["NhaloNode"], dtype=np.int32)
    nfn = np.zeros((NfpTot, Ne, 3), order="F")
    Esc = np.zeros((Np, Ne, 3), order="F")
    Fsc = np.zeros((NfpTot, Ne), order="F")
    pos = np.zeros((Np, Ne, 3), order="F")
    x1D = _f64(x1D)
    _check(lib().sdg_mesh_setup(NeX, NeY, NeZ, p, dom[0], dom[1], dom[2], _p(x1D),
                                _p(VMapM), _p(VMapP), _p(hmap), _p(nfn), _p(Esc),
                                _p(Fsc), _p(pos)))
    Nq = p + 1
    return Mesh(NeX, NeY, NeZ, p, Nq, Np, Nq * Nq, NfpTot, Ne, s["Nhalo"], s["NeA"],
                s["NhaloNode"], VMapM, VMapP, hmap, nfn, Esc, Fsc, pos)


def box_fields(NeX, NeY, NeZ, p, x1D, ic_kind=1, seed=0, vel_kind=0, vel=(1.0, 1.0, 1.0)):
    """Initial q, u, v, w (Np, Ne) of the periodic unit box without building
    the mesh tables (sdg_box_fields: the same values as init_fields on
    mesh_setup's positions)."""
    s = mesh_sizes(NeX, NeY, NeZ, p)
    Np, Ne = s["Np"], s["Ne"]
    q, u, v, w = (np.empty((Np, Ne), order="F") for _ in range(4))
    _check(lib().sdg_box_fields(NeX, NeY, NeZ, p, _p(_f64(x1D)), ic_kind, seed, vel_kind,
                                vel[0], vel[1], vel[2], _p(q), _p(u), _p(v), _p(w)))
    return q, u, v, w


def update_halo(f, mesh):
    """update_halo (mod_mesh.f90:209-221) on a host array, in place."""
    if not (isinstance(f, np.ndarray) and f.dtype == np.float64 and
            (f.flags.f_contiguous or f.flags.c_contiguous and f.ndim == 1)):
        raise SdgError(SDG_ERR_ARG, "update_halo needs a contiguous float64 array")
    _check(lib().sdg_update_halo_host(_p(f), mesh.Np, mesh.Ne, mesh.NhaloNode,
                                      _p(mesh.halo_src_map)))
    return f


def init_fields(mesh, ic_kind=0, seed=0, vel_kind=0, vel=(1.0, 1.0, 1.0)):
    """Initial q,u,v,w(Np,NeA) with halos filled (main.f90:146-162)."""
    shape = (mesh.Np, mesh.NeA)
    q, u, v, w = (np.zeros(shape, order="F") for _ in range(4))
    _check(lib().sdg_init_fields(ic_kind, seed, vel_kind, vel[0], vel[1], vel[2],
                                 _p(mesh.pos_en), mesh.Np, mesh.Ne, _p(q), _p(u),
                                 _p(v), _p(w)))
    for f in (q, u, v, w):
        update_halo(f, mesh)
    return q, u, v, w


def random_velocity(seed):
    out = np.zeros(3)
    _check(lib().sdg_random_velocity(seed, _p(out)))
    return out


def lgl_weights(x1D):
    """LGL quadrature weights w_i = 2 / (N (N+1) P_N(x_i)^2), N = Nq-1."""
    N = len(x1D) - 1
    PN = np.polynomial.legendre.legval(np.asarray(x1D), [0] * N + [1])
    return 2.0 / (N * (N + 1) * PN ** 2)


# ---------------------------------------------------------------------------
# Handle
# ---------------------------------------------------------------------------
class Handle:
    """Operators and mesh resident on the GPU (sdg_init ... sdg_finalize)."""

    def __init__(self, ops, mesh, flags=0):
        self._h = ctypes.c_void_p()
        self.ops, self.mesh, self.flags = ops, mesh, flags
        m = mesh
        _check(lib().sdg_init(ctypes.byref(self._h), m.Nq, m.Np, m.NfpTot, m.Ne, m.NeA,
                              m.NhaloNode, _p(_f64(ops.D1D)), _p(_f64(ops.Lift_mat)),
                              _p(_i32(m.VMapM)), _p(_i32(m.VMapP)),
                              _p(_i32(m.halo_src_map)), _p(_f64(m.normal_fn)),
                              _p(_f64(m.Escale)), _p(_f64(m.Fscale)), flags))

    @property
    def ptr(self):
        return self._h

    def close(self):
        if self._h:
            _check(lib().sdg_finalize(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def cal_tend(self, q, u, v, w, dqdt=None):
        """Drop-in tendency on host arrays (Np,NeA) -> dqdt (Np,NeA)."""
        m = self.mesh
        shape = (m.Np, m.NeA)
        q, u, v, w = (_f64(a, shape) for a in (q, u, v, w))
        if dqdt is None:
            dqdt = np.zeros(shape, order="F")
        _check(lib().sdg_cal_tend(self._h, _p(dqdt), _p(q), _p(u), _p(v), _p(w)))
        return dqdt

    def cal_tend_dev(self, dqdt, q, u, v, w, stream=None):
        """Tendency on device tensors (anything with data_ptr())."""
        _check(lib().sdg_cal_tend_dev(self._h, dqdt.data_ptr(), q.data_ptr(), u.data_ptr(),
                                      v.data_ptr(), w.data_ptr(), stream))

    def update_halo_dev(self, f, stream=None):
        _check(lib().sdg_update_halo_dev(self._h, f.data_ptr(), stream))

    def set_field(self, which, host):
        if not (isinstance(host, np.ndarray) and host.dtype == np.float64 and
                (host.flags.c_contiguous or host.flags.f_contiguous)):
            host = _f64(host)
        if host.size < self.mesh.Np * self.mesh.Ne:
            raise SdgError(SDG_ERR_ARG, "field smaller than (Np, Ne)")
        _check(lib().sdg_set_field(self._h, which, _p(host)))

    def set_state(self, q, u, v, w):
        for which, a in zip((FIELD_Q, FIELD_U, FIELD_V, FIELD_W), (q, u, v, w)):
            self.set_field(which, a)

    def get_field(self, which=FIELD_Q, out=None):
        """Field (Np, Ne) into `out` (any contiguous float64 array of that
        size, e.g. a pinned buffer) or a new array."""
        if out is None:
            out = np.zeros((self.mesh.Np, self.mesh.Ne), order="F")
        elif out.dtype != np.float64 or out.size < self.mesh.Np * self.mesh.Ne or not (
                out.flags.c_contiguous or out.flags.f_contiguous):
            raise SdgError(SDG_ERR_ARG, "get_field: bad output array")
        _check(lib().sdg_get_field(self._h, which, _p(out)))
        return out

    def rk3_steps(self, dt, nsteps):
        _check(lib().sdg_rk3_steps(self._h, dt, nsteps))

    def rk3_steps_host(self, q, dt, nsteps):
        """set_field(q) + rk3_steps(dt, nsteps) + get_field(out=q) in one
        pipelined call (sdg_rk3_steps_host): q, a contiguous float64 array
        of at least Np*Ne values (pinned for the copies to overlap), is
        updated in place."""
        if not (isinstance(q, np.ndarray) and q.dtype == np.float64 and
                (q.flags.c_contiguous or q.flags.f_contiguous) and q.flags.writeable):
            raise SdgError(SDG_ERR_ARG, "rk3_steps_host: q must be a writable contiguous "
                           "float64 array")
        if q.size < self.mesh.Np * self.mesh.Ne:
            raise SdgError(SDG_ERR_ARG, "field smaller than (Np, Ne)")
        _check(lib().sdg_rk3_steps_host(self._h, _p(q), dt, nsteps))
        return q

    def rk3_stage(self, stage, dt):
        """One stage (1..3) of an RK3 step, without a graph."""
        _check(lib().sdg_rk3_stage(self._h, stage, dt))

    def stream(self):
        """The handle's cudaStream_t as an integer."""
        s = ctypes.c_void_p()
        _check(lib().sdg_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def synchronize(self):
        _check(lib().sdg_synchronize(self._h))

    def minmax(self):
        mn, mx = ctypes.c_double(), ctypes.c_double()
        _check(lib().sdg_minmax(self._h, ctypes.byref(mn), ctypes.byref(mx)))
        return mn.value, mx.value

    def diagnostics(self, lgl_w, jac):
        w = _f64(lgl_w)
        mass, l2 = ctypes.c_double(), ctypes.c_double()
        _check(lib().sdg_diagnostics(self._h, _p(w), jac, ctypes.byref(mass),
                                     ctypes.byref(l2)))
        return mass.value, l2.value

    def field_dev_ptr(self, which):
        p = ctypes.c_void_p()
        _check(lib().sdg_field_dev_ptr(self._h, which, ctypes.byref(p)))
        return p.value

    def resident_array(self, which):
        """A resident (Np, NeA) device array as a flat torch tensor view (no
        copy): FIELD_Q, FIELD_U/V/W (compute precision) or ARRAY_STAGE2/3."""
        import torch
        p, es = ctypes.c_void_p(), ctypes.c_int()
        _check(lib().sdg_resident_array(self._h, which, ctypes.byref(p), ctypes.byref(es)))
        n = self.mesh.Np * self.mesh.NeA
        return _device_view(p.value, n, torch.float64 if es.value == 8 else torch.float32)

    def stage_input(self, stage):
        """The input array of RK stage 1..3 (see resident_array)."""
        return self.resident_array((FIELD_Q, ARRAY_STAGE2, ARRAY_STAGE3)[stage - 1])

    def update_halo_stage(self, stage):
        """update_halo of stage `stage`'s input on the handle's stream."""
        _check(lib().sdg_update_halo_stage(self._h, stage))

    def timers(self):
        t = np.zeros(4)
        _check(lib().sdg_timers(self._h, _p(t)))
        return t

    def launch_count(self):
        return int(lib().sdg_launch_count(self._h))

    def set_kernel_variant(self, variant):
        """0 automatic, 1 one tile per block, 2 persistent bulk-copy ring,
        3 one tile per block at 8 blocks per SM, 4 bulk-copy ring with split
        columns (orders with one element per tile)."""
        _check(lib().sdg_set_kernel_variant(self._h, variant))

    def inject_wait_timeout(self, tile, spins=0):
        """Test hook: the pipelined kernel skips the copies of element tile
        `tile`, so its bounded wait runs out after `spins` polls and the next
        synchronising call raises; tile < 0 turns it off."""
        _check(lib().sdg_debug_inject_wait_timeout(self._h, tile, spins))


def chunk_bounds(Ne, Np, reach):
    """Element-chunk boundaries of the host-buffer calls for Ne elements of
    Np nodes whose face neighbours lie within cyclic index distance `reach`
    (host logic, no device needed); empty when the mesh does not pipeline."""
    e0 = np.zeros(64, dtype=np.int32)
    n = ctypes.c_int(0)
    _check(lib().sdg_debug_chunk_bounds(Ne, Np, reach, _p(e0), e0.size, ctypes.byref(n)))
    return e0[: n.value + 1] if n.value else e0[:0]


def step_plan(nbr, uploads, steps=1):
    """Launch order of `steps` chunked RK steps over len(nbr) chunks with
    neighbour lists nbr (host logic): rows (stage 0 .. 3*steps-1, first
    chunk, last chunk, upload waited for or -1)."""
    S = len(nbr)
    ptr = np.zeros(S + 1, dtype=np.int32)
    ptr[1:] = np.cumsum([len(l) for l in nbr])
    idx = np.array([c for l in nbr for c in l] or [0], dtype=np.int32)
    ops = np.zeros(4 * 3 * steps * S, dtype=np.int32)
    n = ctypes.c_int(0)
    _check(lib().sdg_debug_step_plan(S, _p(ptr), _p(idx), steps, int(bool(uploads)),
                                     _p(ops), ops.size, ctypes.byref(n)))
    return ops[: 4 * n.value].reshape(-1, 4)


def _device_view(ptr, n, dtype):
    """A torch tensor over n elements of device memory at ptr (no copy,
    not owned: the library keeps the allocation)."""
    import torch

    class _Arr:
        pass

    a = _Arr()
    a.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8" if dtype == torch.float64
                                  else "<f4", "data": (ptr, False), "version": 3,
                                  "strides": None}
    return torch.as_tensor(a, device="cuda")


# ---------------------------------------------------------------------------
# The reference's operator/driver surface
# ---------------------------------------------------------------------------
_EVALTYPES = {"GPU": 0, "OPT1": FLAG_EXACT, "GENERAL": FLAG_EXACT | FLAG_ORDER_GENERAL}
_eval_flags = None
_handles = {}


def dg_optr_kernel_setup(evaltype):
    """Selector of mod_dg_optr_kernel.f90:45-58.  Unknown types raise (the
    reference only prints and leaves the type unset, kern:54-55)."""
    global _eval_flags
    key = str(evaltype).strip().upper()
    if key not in _EVALTYPES:
        raise SdgError(SDG_ERR_ARG, f"Unsupported dgoptr_evaltype: {evaltype}")
    _eval_flags = _EVALTYPES[key]


def advect3d_eq_cal_tend(dqdt, q, u, v, w, D1D, D1D_tr, Lift_mat, VMapM, VMapP,
                         normal_fn, Escale, Fscale, Nq, Np, NfpTot, Ne, NeA,
                         halo_src_map=None):
    """advect3d_eq_cal_tend (mod_advect3d_eq.f90:41-85) on the GPU.

    Same arguments and meaning as the reference: writes dqdt(:,1:Ne) from
    q,u,v,w(Np,NeA), reading the plus side through VMapP (halo included).
    The device tables are built on first use for a given mesh and cached.
    """
    if _eval_flags is None:
        raise SdgError(SDG_ERR_STATE, "call dg_optr_kernel_setup first")
    if D1D_tr is not None and not np.array_equal(np.asarray(D1D_tr), np.asarray(D1D).T):
        raise SdgError(SDG_ERR_ARG, "D1D_tr is not the transpose of D1D")
    key = (id(VMapM), id(VMapP), id(Lift_mat), id(D1D), Nq, Ne, NeA, _eval_flags)
    h = _handles.get(key)
    if h is None:
        NhaloNode = 0 if halo_src_map is None else int(np.asarray(halo_src_map).size)
        ops = Operators(Nq - 1, Nq, None, _f64(D1D), None, _f64(Lift_mat))
        mesh = Mesh(None, None, None, Nq - 1, Nq, Np, Nq * Nq, NfpTot, Ne, None, NeA,
                    NhaloNode, _i32(VMapM), _i32(VMapP),
                    _i32(halo_src_map if halo_src_map is not None else np.zeros(0)),
                    _f64(normal_fn), _f64(Escale), _f64(Fscale), None)
        h = Handle(ops, mesh, _eval_flags)
        _handles[key] = (h, (VMapM, VMapP, Lift_mat, D1D))
    else:
        h = h[0]
    out = h.cal_tend(q, u, v, w)
    dqdt[:, :Ne] = out[:, :Ne]
    return dqdt


def divlike_dirXYZ_var_dev(D1D, nvar, Ne, in_x, in_y, in_z, out_x, out_y, out_z, flags=0,
                           stream=None):
    """element_operation_kernel_matvec_divlike_dirXYZ_var5_P<p>
    (mod_dg_optr_kernel_opt1.F90.erb:347-465) on device tensors.

    The arrays (anything with data_ptr(), float64, contiguous) hold element
    e, field v, node n = i + Nq*j + Nq^2*k at n + Np*(v + nvar*e); out_d
    receives the d-derivative of in_d.  D1D is the (Nq,Nq) operator matrix.
    flags: 0, FLAG_EXACT, or FLAG_EXACT | FLAG_ORDER_GENERAL."""
    D = _f64(D1D)
    _check(lib().sdg_divlike_dev(D.shape[0], nvar, Ne, _p(D), in_x.data_ptr(), in_y.data_ptr(),
                                 in_z.data_ptr(), out_x.data_ptr(), out_y.data_ptr(),
                                 out_z.data_ptr(), flags, stream))


def gradlike_dirXYZ_dev(D1D, Ne, vec_in, out_x, out_y, out_z, flags=0, stream=None):
    """element_operation_kernel_matvec_gradlike_dirXYZ_P<p>
    (mod_dg_optr_kernel_opt1.F90.erb:166-219) on device tensors: the x-, y-
    and z-derivatives of one field (layout as divlike_dirXYZ_var_dev with
    nvar = 1)."""
    D = _f64(D1D)
    _check(lib().sdg_gradlike_dev(D.shape[0], Ne, _p(D), vec_in.data_ptr(), out_x.data_ptr(),
                                  out_y.data_ptr(), out_z.data_ptr(), flags, stream))


class Problem:
    """Operators + mesh + handle for a periodic unit-cube run."""

    def __init__(self, NeX, NeY, NeZ, p, flags=0, opdir=OPERATOR_DIR):
        self.ops = read_operators(p, opdir)
        self.mesh = mesh_setup(NeX, NeY, NeZ, p, self.ops.x1D)
        self.handle = Handle(self.ops, self.mesh, flags)

    def close(self):
        self.handle.close()


# ---------------------------------------------------------------------------
# Batched ensembles and the serving loop
# ---------------------------------------------------------------------------
class Batch:
    """Many periodic-box instances advanced together (sdg_batch_*)."""

    def __init__(self, flags=0):
        self._b = ctypes.c_void_p()
        _check(lib().sdg_batch_create(ctypes.byref(self._b), flags))
        self.shapes = []

    def add(self, NeX, NeY, NeZ, p, ops, q, u, v, w, dt):
        """Adds an instance; q,u,v,w are (Np, Ne) or (Np, NeA) arrays."""
        n = (p + 1) ** 3 * NeX * NeY * NeZ
        arrs = [_f64(a).reshape(-1, order="F")[:n].copy() for a in (q, u, v, w)]
        i = ctypes.c_int()
        _check(lib().sdg_batch_add(self._b, NeX, NeY, NeZ, p, _p(_f64(ops.D1D)),
                                   _p(_f64(ops.Lift_mat)), *[_p(a) for a in arrs], dt,
                                   ctypes.byref(i)))
        self.shapes.append(((p + 1) ** 3, NeX * NeY * NeZ))
        return i.value

    def commit(self, autotune=True):
        _check(lib().sdg_batch_commit(self._b, 1 if autotune else 0))

    def run(self, nsteps):
        _check(lib().sdg_batch_run(self._b, nsteps))

    def get(self, i):
        np_, ne = self.shapes[i]
        out = np.zeros((np_, ne), order="F")
        _check(lib().sdg_batch_get(self._b, i, _p(out)))
        return out

    def info(self):
        buf = np.zeros(512)
        n = lib().sdg_batch_info(self._b, _p(buf), 512)
        v = buf[:n]
        groups = []
        for g in range(int(v[4])):
            r = v[5 + 8 * g: 13 + 8 * g]
            groups.append({"p": int(r[0]), "mixed": bool(r[1]), "tiles": int(r[2]),
                           "variant": int(r[3]), "ms_pipe": r[4], "ms_block": r[5],
                           "ms_block8": r[6], "ms_split": r[7]})
        return {"instances": int(v[0]), "dof": int(v[1]), "run_s": v[2],
                "dof_steps": int(v[3]), "groups": groups}

    def inject_wait_timeout(self, tile, spins=0):
        """Test hook: tile `tile` of every group is skipped (see Handle)."""
        _check(lib().sdg_batch_debug_inject_wait_timeout(self._b, tile, spins))

    def close(self):
        if self._b:
            _check(lib().sdg_batch_destroy(self._b))
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SERVE_QUEUED, SERVE_RUNNING, SERVE_DONE, SERVE_FAILED = 0, 1, 2, 3


class Server:
    """The serving loop (sdg_serve_*): submit requests, poll, fetch results."""

    def __init__(self, max_bytes=0.0):
        self._s = ctypes.c_void_p()
        _check(lib().sdg_serve_create(ctypes.byref(self._s), float(max_bytes)))
        self.shapes = {}

    def submit(self, NeX, NeY, NeZ, p, ops, q, u, v, w, dt, nsteps, mixed=False):
        n = (p + 1) ** 3 * NeX * NeY * NeZ
        arrs = [np.ascontiguousarray(_f64(a).reshape(-1, order="F")[:n]) for a in (q, u, v, w)]
        i = ctypes.c_int()
        _check(lib().sdg_serve_submit(self._s, NeX, NeY, NeZ, p, _p(_f64(ops.D1D)),
                                      _p(_f64(ops.Lift_mat)), *[_p(a) for a in arrs], dt,
                                      nsteps, FLAG_MIXED if mixed else 0, ctypes.byref(i)))
        self.shapes[i.value] = ((p + 1) ** 3, NeX * NeY * NeZ)
        return i.value

    def poll(self, i):
        st = ctypes.c_int()
        t = np.zeros(2)
        _check(lib().sdg_serve_poll(self._s, i, ctypes.byref(st), _p(t)))
        return st.value, t[0], t[1]

    def result(self, i):
        np_, ne = self.shapes[i]
        out = np.zeros((np_, ne), order="F")
        _check(lib().sdg_serve_result(self._s, i, _p(out)))
        return out

    def wait(self, timeout_s=0.0):
        _check(lib().sdg_serve_wait(self._s, float(timeout_s)))

    def stats(self):
        out = np.zeros(4)
        _check(lib().sdg_serve_stats(self._s, _p(out)))
        return {"busy_s": out[0], "dof_steps": out[1], "iterations": int(out[2]),
                "bytes_in_use": out[3]}

    def close(self):
        if self._s:
            _check(lib().sdg_serve_destroy(self._s))
            self._s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
