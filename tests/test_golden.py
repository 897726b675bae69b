"""The oracle and the library's host set-up against golden fixtures produced
from the reference's own source (tests/golden/make_golden.py evaluates the
Fortran files through a mechanical translator).  Bit-exact throughout.

The GPU half (exact kernels and the sdg_run driver against the same
fixtures) is in test_gpu_golden.py.
"""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import orc
import sdg_b200 as sdg

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from golden_inputs import MAIN_CASES, MESH_CASES, TEND_CASES, tend_inputs  # noqa: E402


@pytest.fixture(scope="module")
def gold(built):
    return np.load(os.path.join(GOLDEN, "golden.npz"))


def main_lines():
    text = open(os.path.join(GOLDEN, "golden_main.txt")).read().split("\n")
    out, cur = {}, None
    for ln in text:
        if ln.startswith("== "):
            cur = ln[3:]
            out[cur] = []
        elif cur and re.match(r"^\s*\d+\s+\S+\s+\S+$", ln):
            out[cur].append(ln)
    return out


TABLES = {"vmapm": "VMapM", "vmapp": "VMapP", "halo_src_map": "halo_src_map",
          "normal_fn": "normal_fn", "escale": "Escale", "fscale": "Fscale",
          "pos_en": "pos_en"}


@pytest.mark.parametrize("NeX,NeY,NeZ,p", MESH_CASES)
def test_mesh_tables_match_golden(gold, NeX, NeY, NeZ, p):
    x1D = orc.read_operators(p).x1D
    o = orc.mesh_setup(NeX, NeY, NeZ, p, x1D)
    s = sdg.mesh_setup(NeX, NeY, NeZ, p, x1D)
    for k, attr in TABLES.items():
        g = gold[f"mesh_{NeX}x{NeY}x{NeZ}_p{p}/{k}"]
        assert np.array_equal(getattr(o, attr), g.reshape(getattr(o, attr).shape)), k
        assert np.array_equal(getattr(s, attr), g.reshape(getattr(s, attr).shape)), k


def golden_case_inputs(p, dims):
    ops = orc.read_operators(p)
    m = orc.mesh_setup(*dims, p, ops.x1D)
    fields = [np.asfortranarray(x) for x in tend_inputs(p, dims, m.Np, m.NeA)]
    for f in fields:
        orc.update_halo(f, m)
    return ops, m, fields


@pytest.mark.parametrize("kind,p,dims", TEND_CASES)
def test_oracle_tendency_matches_golden(gold, kind, p, dims):
    ops, m, (q, u, v, w) = golden_case_inputs(p, dims)
    ev = orc.OPT1 if kind == "OPT1" else orc.GENERAL
    got = orc.cal_tend(ev, q, u, v, w, ops, m)[:, : m.Ne]
    assert np.array_equal(got, gold[f"tend_{kind}_p{p}"])


def conf_params(text):
    d = {}
    for k, v in re.findall(r"(\w+)\s*=\s*([^,\n!]+)", text):
        d[k.lower()] = v.strip().strip('"')
    return d


@pytest.mark.parametrize("name", sorted(MAIN_CASES))
def test_oracle_program_matches_golden(gold, name, tmp_path):
    """The oracle CLI on the same namelist prints the same lines as the
    reference's main program, and ends in the same state."""
    conf = tmp_path / "input.conf"
    conf.write_text(MAIN_CASES[name])
    r = subprocess.run([orc.CLI_PATH, str(conf), orc.OPERATOR_DIR],
                       capture_output=True, text=True, check=True)
    got = [ln for ln in r.stdout.split("\n") if re.match(r"^\s*\d+\s+\S+\s+\S+$", ln)]
    assert got == main_lines()[name]
    prm = conf_params(MAIN_CASES[name])
    dims = [int(prm.get(k, 4)) for k in ("nex", "ney", "nez")]
    p = int(prm["polyorder"])
    vel = tuple(float(prm.get(k, "1.0").lower().replace("d", "e"))
                for k in ("vel_x", "vel_y", "vel_z"))
    ops = orc.read_operators(p)
    m = orc.mesh_setup(*dims, p, ops.x1D)
    q, u, v, w = orc.init_fields(m, ic_kind=0, vel_kind=0, vel=vel)
    ev = orc.OPT1 if prm["dgoptrkernel_opttype"].upper() == "OPT1" else orc.GENERAL
    dt = float(prm["dt"].lower().replace("d", "e"))
    orc.run_rk3(ev, q, u, v, w, ops, m, dt, int(prm["nstep"]))
    assert np.array_equal(q[:, : m.Ne], gold[f"main_{name}/q"])
