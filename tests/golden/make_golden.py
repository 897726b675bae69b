"""Generates the golden fixtures of tests/golden/ from the reference source.

Run in the build container (it reads the reference checkout, which the GPU
box does not have):

    python tests/golden/make_golden.py /path/to/scale-dg-kernel-extraction

Each case is produced by evaluating the reference's own Fortran files through
f90eval (a mechanical translator; no Fortran compiler exists in the image):

  mesh_<NeX>x<NeY>x<NeZ>_p<p>   mesh_setup tables (VMapM, VMapP,
                                halo_src_map, normal_fn, Escale, Fscale, pos_en)
  tend_<kind>_p<p>              advect3d_eq_cal_tend on seeded inputs, after
                                dg_optr_kernel_setup("GENERAL"/"OPT1"),
                                dqdt(:,1:Ne)
  main_<name>                   the main program on a namelist file: the
                                printed "istep min max" lines and q(:,1:Ne)

Inputs of the tendency cases come from golden_inputs.splitmix_field, which
the tests recompute bit for bit.  Output: golden.npz (+ golden_main.txt).
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import f90eval as fe  # noqa: E402
from golden_inputs import TEND_CASES, MESH_CASES, MAIN_CASES, tend_inputs  # noqa: E402

FILES = ["mod_common.f90", "mod_mesh.f90", "mod_dg_optr_kernel_opt1.f90",
         "mod_dg_optr_kernel.f90", "mod_advect3d_eq.f90", "main.f90"]


def interp(ref, argv=()):
    return fe.Interp([os.path.join(ref, f) for f in FILES], ref, argv)


def mesh_case(ref, NeX, NeY, NeZ, p):
    I = interp(ref)
    args = [NeX, NeY, NeZ, p, 1.0, 1.0, 1.0]
    I.call("mesh_setup", [(lambda a=a: a) for a in args], None)
    M = I.MOD["mod_mesh"]
    out = {}
    for name in ("vmapm", "vmapp", "halo_src_map", "normal_fn", "escale", "fscale",
                 "pos_en"):
        a = M[name]
        out[name] = a.flat().copy().reshape(a.dims, order="F")
    return I, out


def tend_case(ref, kind, p, dims):
    I, _ = mesh_case(ref, *dims, p)
    M = I.MOD["mod_mesh"]
    I.call("dg_optr_kernel_setup", [lambda: kind], None)
    Np, NeA, Ne = M["np"], M["nea"], M["ne"]
    fields = tend_inputs(p, dims, Np, NeA)
    arrs = []
    for f in fields:
        a = fe.FArr.zeros((Np, NeA), np.float64)
        a.flat()[:] = f.reshape(-1, order="F")
        I.call("update_halo", [lambda a=a: a], [("array", a)])
        arrs.append(a)
    dqdt = fe.FArr.zeros((Np, NeA), np.float64)
    actual = [dqdt] + arrs + [M["d1d"], M["d1d_tr"], M["lift_mat"], M["vmapm"],
                              M["vmapp"], M["normal_fn"], M["escale"], M["fscale"]]
    scal = [M["nq"], Np, M["nfptot"], Ne, NeA]
    thunks = [(lambda a=a: a) for a in actual + scal]
    refs = [("array", a) for a in actual] + [None] * len(scal)
    I.call("advect3d_eq_cal_tend", thunks, refs)
    return dqdt.flat().copy().reshape(Np, NeA, order="F")[:, :Ne]


def main_case(ref, conf_text):
    with tempfile.TemporaryDirectory() as td:
        conf = os.path.join(td, "input.conf")
        with open(conf, "w") as f:
            f.write(conf_text)
        I = interp(ref, [conf])
        lines = fe.run_program(I)
        V = I.HOST["main"]
        q = V["q"]
        Np, Ne = I.MOD["mod_mesh"]["np"], I.MOD["mod_mesh"]["ne"]
        return lines, q.flat().copy().reshape(q.dims, order="F")[:, :Ne].copy()


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SDG_REFERENCE")
    if not ref or not os.path.isdir(ref):
        sys.exit("usage: make_golden.py <reference checkout>")
    out = {}
    for NeX, NeY, NeZ, p in MESH_CASES:
        _, tabs = mesh_case(ref, NeX, NeY, NeZ, p)
        for k, v in tabs.items():
            out[f"mesh_{NeX}x{NeY}x{NeZ}_p{p}/{k}"] = v
        print("mesh", NeX, NeY, NeZ, p, flush=True)
    for kind, p, dims in TEND_CASES:
        out[f"tend_{kind}_p{p}"] = tend_case(ref, kind, p, dims)
        print("tend", kind, p, dims, flush=True)
    text = []
    for name, conf in MAIN_CASES.items():
        lines, q = main_case(ref, conf)
        out[f"main_{name}/q"] = q
        text.append(f"== {name}")
        text.extend(lines)
        print("main", name, flush=True)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    with open(os.path.join(HERE, "golden_main.txt"), "w") as f:
        f.write("\n".join(text) + "\n")


if __name__ == "__main__":
    main()
