"""The Fortran side of the drop-in (CPU only).

* Every bind(C) interface of fortran/mod_dg_gpu.f90 matches its prototype in
  include/sdg_gpu.h: the C name, the number of arguments, and per argument
  the type and whether it is passed by value or by reference.
* The reference-side patch (fortran/reference_gpu_option.patch: the "GPU"
  case of dg_optr_kernel_setup, mod_dg_optr_kernel.f90:45-58; the GPU branch
  of advect3d_eq_cal_tend, mod_advect3d_eq.f90:41-85; the set-up and the
  resident time loop of main.f90:51-80, 132-139; the halo map export of
  mod_mesh.f90:66-68; the Makefile) applies cleanly to the reference
  sources and calls only what mod_dg_gpu.f90 makes public.

No Fortran compiler exists in this image, so neither file is compiled here;
these checks catch drift between the binding, the patch and the C header.
"""
import os
import re
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FORTRAN = os.path.join(REPO, "scale-dg-kernel-extraction_b200", "fortran")
MODULE = os.path.join(FORTRAN, "mod_dg_gpu.f90")
PATCH = os.path.join(FORTRAN, "reference_gpu_option.patch")
HEADER = os.path.join(REPO, "include", "sdg_gpu.h")
REFERENCE = "/root/reference"


def c_prototypes():
    """name -> (return type, [(type, is_pointer_level)]) from the header."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    protos = {}
    for m in re.finditer(r"([A-Za-z_][\w \*]*?)\b(sdg_\w+)\s*\(([^;{]*?)\)\s*;", text):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3)
        params = []
        for a in [x.strip() for x in args.split(",") if x.strip() and x.strip() != "void"]:
            stars = a.count("*")
            base = re.sub(r"\bconst\b", "", a.replace("*", " ")).split()
            # drop the parameter name
            base = base[:-1] if len(base) > 1 else base
            params.append((" ".join(base), stars))
        protos[name] = (ret, params)
    return protos


def fortran_interfaces():
    """C name -> [(fortran type, has value)] in dummy-argument order."""
    text = open(MODULE).read()
    text = re.sub(r"!.*", "", text)
    text = re.sub(r"&\s*\n\s*", " ", text)
    out = {}
    for m in re.finditer(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\s*\(\s*C\s*,\s*name\s*=\s*"
                         r"\"(\w+)\"\s*\)(.*?)end function", text, flags=re.S | re.I):
        fname, dummies, cname, body = m.groups()
        names = [d.strip().lower() for d in dummies.split(",") if d.strip()]
        decl = {}
        for line in body.split("\n"):
            if "::" not in line:
                continue
            lhs, rhs = line.split("::", 1)
            ftype = lhs.split(",")[0].strip().lower().replace(" ", "")
            value = "value" in lhs.lower()
            for var in re.split(r",(?![^()]*\))", rhs):
                v = re.sub(r"\(.*\)", "", var).strip().lower()
                if v:
                    decl[v] = (ftype, value)
        out[cname] = [decl[n] for n in names]
    return out


# C parameter (type, pointer level) -> the Fortran dummy it must be.
def expected(ctype, stars):
    if stars == 0:
        return {"int": ("integer(c_int)", True), "double": ("real(c_double)", True),
                "longlong": ("integer(c_long_long)", True)}[ctype.replace(" ", "")]
    if stars == 1:
        if ctype in ("void", "sdg_handle", "sdg_batch", "sdg_server"):
            return ("type(c_ptr)", True)
        return {"int": ("integer(c_int)", False), "double": ("real(c_double)", False),
                "char": ("character(kind=c_char)", False)}[ctype]
    if stars == 2:
        return ("type(c_ptr)", False)
    raise AssertionError((ctype, stars))


def test_bind_c_interfaces_match_header():
    protos = c_prototypes()
    ifaces = fortran_interfaces()
    assert len(ifaces) >= 10, sorted(ifaces)
    for cname, dummies in ifaces.items():
        assert cname in protos, f"{cname} is not declared in include/sdg_gpu.h"
        ret, params = protos[cname]
        assert ret == "int", (cname, ret)
        assert len(dummies) == len(params), (cname, len(dummies), len(params))
        for k, ((ctype, stars), got) in enumerate(zip(params, dummies)):
            ok = {expected(ctype, stars)}
            if stars == 1:
                # A device address (or any pointer) may travel as a C
                # address by value: the same ABI as an array by reference.
                ok.add(("type(c_ptr)", True))
            assert got in ok, (cname, k, ctype, stars, got)


def test_module_declares_the_resident_path():
    ifaces = fortran_interfaces()
    for name in ("sdg_init", "sdg_finalize", "sdg_cal_tend", "sdg_set_field",
                 "sdg_get_field", "sdg_rk3_steps", "sdg_minmax", "sdg_last_error"):
        assert name in ifaces, name


@pytest.mark.skipif(not os.path.isdir(REFERENCE) or shutil.which("patch") is None,
                    reason="needs the reference sources and patch(1)")
def test_reference_patch_applies_and_uses_public_names(tmp_path):
    for f in ("Makefile", "main.f90", "mod_advect3d_eq.f90", "mod_dg_optr_kernel.f90",
              "mod_mesh.f90"):
        shutil.copy(os.path.join(REFERENCE, f), tmp_path / f)
    r = subprocess.run(["patch", "-p1", "--forward", "-i", PATCH], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert ".rej" not in r.stdout
    module = open(MODULE).read().lower()
    public = set()
    for m in re.finditer(r"public\s*::([^\n]*)", module):
        public |= {x.strip() for x in m.group(1).split(",")}
    patched = "".join(open(tmp_path / f).read().lower()
                      for f in ("main.f90", "mod_advect3d_eq.f90"))
    used = set(re.findall(r"\b(dg_gpu_\w+)", patched))
    assert used and used <= public, used - public
    sel = open(tmp_path / "mod_dg_optr_kernel.f90").read()
    assert 'case ("GPU")' in sel and "error stop" in sel
