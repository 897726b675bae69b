"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/sdg_gpu.h declares, validates arguments and mesh tables with the
documented status codes, and fails loudly (no CPU path) without a device.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import orc
import sdg_b200 as sdg

HEADER = os.path.join(os.path.dirname(sdg.PKG_DIR), "include", "sdg_gpu.h")


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sdg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = sdg.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
        assert n in sdg.SIGNATURES, f"{n} has no binding"
    out = subprocess.run(["nm", "-D", "--defined-only", sdg.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (sdg_\w+)", out))
    assert set(names) <= exported


def test_version():
    assert sdg.lib().sdg_version().decode().count(".") == 2


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_operator_errors(tmp_path):
    with pytest.raises(sdg.SdgError) as e:
        sdg.read_operators(16)
    assert e.value.code == sdg.SDG_ERR_ARG
    with pytest.raises(sdg.SdgError) as e:
        sdg.read_operators(3, str(tmp_path))
    assert e.value.code == sdg.SDG_ERR_IO
    src = os.path.join(sdg.OPERATOR_DIR, "p3.dat")
    data = open(src).read()
    (tmp_path / "p3.dat").write_text(data[: len(data) // 2])
    with pytest.raises(sdg.SdgError) as e:
        sdg.read_operators(3, str(tmp_path))
    assert e.value.code == sdg.SDG_ERR_IO
    (tmp_path / "p3.dat").write_text(data.replace("E", "Q", 5))
    with pytest.raises(sdg.SdgError) as e:
        sdg.read_operators(3, str(tmp_path))
    assert e.value.code == sdg.SDG_ERR_IO


def test_mesh_size_errors():
    with pytest.raises(sdg.SdgError) as e:
        sdg.mesh_sizes(0, 4, 4, 3)
    assert e.value.code == sdg.SDG_ERR_ARG
    with pytest.raises(sdg.SdgError) as e:   # Np*NeA overflows int32
        sdg.mesh_sizes(256, 256, 256, 7)
    assert "int32" in str(e.value)
    s = sdg.mesh_sizes(32, 32, 32, 7)
    assert s == {"Ne": 32768, "Nhalo": 6144, "NeA": 38912, "NhaloNode": 393216,
                 "Np": 512, "NfpTot": 384}


def _tables(p=2, dims=(3, 2, 2)):
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(*dims, p, ops.x1D)
    return ops, mesh


@pytest.mark.parametrize("corrupt", ["vmapm", "vmapp", "vmapp_halo", "normal",
                                     "fscale", "escale", "hmap"])
def test_init_rejects_unstructured_tables(corrupt):
    ops, m = _tables()
    m = m._replace(VMapM=m.VMapM.copy(order="F"), VMapP=m.VMapP.copy(order="F"),
                   normal_fn=m.normal_fn.copy(order="F"), Fscale=m.Fscale.copy(order="F"),
                   Escale=m.Escale.copy(order="F"), halo_src_map=m.halo_src_map.copy())
    if corrupt == "vmapm":
        m.VMapM[3, 1] += 1
    elif corrupt == "vmapp":
        interior = np.where(m.VMapP[:, 0] <= m.Np * m.Ne)[0]
        i0, i1 = interior[0], interior[1]
        m.VMapP[i0, 0], m.VMapP[i1, 0] = m.VMapP[i1, 0], m.VMapP[i0, 0]
    elif corrupt == "vmapp_halo":
        halo = np.where(m.VMapP[:, 0] > m.Np * m.Ne)[0]
        m.VMapP[halo[1], 0] += 3
    elif corrupt == "normal":
        m.normal_fn[0, 2, 0] = 0.5
    elif corrupt == "fscale":
        m.Fscale[1, 0] *= 2
    elif corrupt == "escale":
        m.Escale[5, 1, 2] *= 2
    elif corrupt == "hmap":
        m.halo_src_map[0] = m.Np * m.Ne + 5
    with pytest.raises(sdg.SdgError) as e:
        sdg.Handle(ops, m)
    assert e.value.code == sdg.SDG_ERR_MESH, str(e.value)


def test_init_argument_errors():
    ops, m = _tables()
    with pytest.raises(sdg.SdgError) as e:
        sdg.Handle(ops, m, flags=sdg.FLAG_MIXED | sdg.FLAG_EXACT)
    assert e.value.code == sdg.SDG_ERR_ARG
    with pytest.raises(sdg.SdgError) as e:
        sdg.Handle(ops, m, flags=64)
    assert e.value.code == sdg.SDG_ERR_ARG
    with pytest.raises(sdg.SdgError):
        sdg.Handle(ops, m._replace(Np=m.Np + 1))


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_cpu_fallback_without_device():
    ops, m = _tables()
    with pytest.raises(sdg.SdgError) as e:
        sdg.Handle(ops, m)
    assert e.value.code == sdg.SDG_ERR_CUDA
    assert "no CUDA device" in str(e.value)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_ensembles_fail_loudly_without_device():
    with pytest.raises(sdg.SdgError) as e:
        sdg.Batch(0)
    assert e.value.code == sdg.SDG_ERR_CUDA
    with pytest.raises(sdg.SdgError) as e:
        sdg.Server()
    assert e.value.code == sdg.SDG_ERR_CUDA


def test_ensemble_argument_errors():
    with pytest.raises(sdg.SdgError) as e:
        sdg.Batch(sdg.FLAG_MIXED | sdg.FLAG_EXACT)
    assert e.value.code == sdg.SDG_ERR_ARG


def test_derivative_operator_argument_errors():
    """sdg_divlike_dev / sdg_gradlike_dev check sizes, flags and arrays before
    touching a device."""
    import ctypes
    L = sdg.lib()
    D = np.eye(4, order="F")
    dp = ctypes.c_void_p(D.ctypes.data)
    one = ctypes.c_void_p(8)  # never dereferenced: every call below fails first
    def div(Nq=4, nvar=5, Ne=2, flags=0, arr=one, d=dp):
        return L.sdg_divlike_dev(Nq, nvar, Ne, d, arr, arr, arr, arr, arr, arr, flags, None)
    assert div(Nq=1) == sdg.SDG_ERR_ARG
    assert div(Nq=17) == sdg.SDG_ERR_ARG
    assert div(nvar=0) == sdg.SDG_ERR_ARG
    assert div(Ne=-1) == sdg.SDG_ERR_ARG
    assert div(flags=sdg.FLAG_MIXED) == sdg.SDG_ERR_ARG
    assert div(flags=sdg.FLAG_ORDER_GENERAL) == sdg.SDG_ERR_ARG
    assert div(arr=None) == sdg.SDG_ERR_ARG
    assert div(d=None) == sdg.SDG_ERR_ARG
    assert L.sdg_gradlike_dev(4, 2, dp, None, one, one, one, 0, None) == sdg.SDG_ERR_ARG
    assert L.sdg_gradlike_dev(0, 2, dp, one, one, one, one, 0, None) == sdg.SDG_ERR_ARG


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_derivative_operators_fail_loudly_without_device():
    import ctypes
    D = np.eye(4, order="F")
    a = np.zeros(64 * 2)
    pa = ctypes.c_void_p(a.ctypes.data)
    rc = sdg.lib().sdg_gradlike_dev(4, 2, ctypes.c_void_p(D.ctypes.data), pa, pa, pa, pa, 0,
                                    None)
    assert rc == sdg.SDG_ERR_CUDA


def test_evaltype_selector():
    with pytest.raises(sdg.SdgError):
        sdg.dg_optr_kernel_setup("FASTEST")
    for t in ("GPU", "OPT1", "GENERAL", " opt1 "):
        sdg.dg_optr_kernel_setup(t)


RUN = os.path.join(sdg.PKG_DIR, "sdg_run")


def _run(args, cwd):
    return subprocess.run([RUN] + args, capture_output=True, text=True, cwd=cwd)


def test_driver_errors(tmp_path):
    if not os.path.exists(RUN):
        subprocess.run(["make", "-s", "-C", sdg.PKG_DIR, "sdg_run"], check=True)
    r = _run([], tmp_path)
    assert r.returncode == 1 and "configuration file argument is required" in r.stderr
    (tmp_path / "bad.conf").write_text("&PARAM_ADVECT3D\n NeX = 4,\n Bogus = 1\n/\n")
    r = _run(["bad.conf"], tmp_path)
    assert r.returncode == 1 and "unknown namelist key BOGUS" in r.stderr
    (tmp_path / "opt.conf").write_text('&PARAM_ADVECT3D\n DGOptrKernel_OptType = "FAST"\n/\n')
    r = _run(["opt.conf"], tmp_path)
    assert r.returncode == 2 and "Unsupported dgoptr_evaltype" in r.stderr
    (tmp_path / "nogroup.conf").write_text("NeX = 4\n")
    r = _run(["nogroup.conf"], tmp_path)
    assert r.returncode == 1 and "not found" in r.stderr
    (tmp_path / "p.conf").write_text("&PARAM_ADVECT3D\n PolyOrder = 16,\n/\n")
    r = _run(["p.conf"], tmp_path)
    assert r.returncode == 1 and "1..15" in r.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_driver_fails_loudly_without_device(tmp_path):
    shutil.copytree(sdg.OPERATOR_DIR, tmp_path / "operator_data")
    (tmp_path / "input.conf").write_text(
        '&PARAM_ADVECT3D\n NeX = 2, NeY = 2, NeZ = 2,\n PolyOrder = 3,\n'
        ' DGOptrKernel_OptType = "GPU" ! new option\n nstep = 2,\n/\n')
    r = _run(["input.conf"], tmp_path)
    assert r.returncode == 1 and "no CUDA device" in r.stderr
