"""GPU kernels and the sdg_run driver against the golden fixtures produced
from the reference's own source (needs a B200).

* The exact kernels (evaltype OPT1 / GENERAL) reproduce the reference's
  tendency bit for bit on every golden case, p = 1..15.
* sdg_run, given the same namelist files as the reference's main program,
  prints identical "istep min max" lines and ends in the identical state.
* The fast kernels ("GPU") stay within 1e-12.
"""
import os
import re
import shutil
import subprocess
import sys

import numpy as np
import pytest

import orc
import sdg_b200 as sdg
from conftest import rel_maxnorm

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from golden_inputs import MAIN_CASES, TEND_CASES, tend_inputs  # noqa: E402
from test_golden import main_lines  # noqa: E402


@pytest.fixture(scope="module")
def gold(built):
    return np.load(os.path.join(GOLDEN, "golden.npz"))


@pytest.mark.parametrize("kind,p,dims", TEND_CASES)
def test_gpu_tendency_matches_golden(gold, kind, p, dims):
    ops = sdg.read_operators(p)
    m = sdg.mesh_setup(*dims, p, ops.x1D)
    fields = [np.asfortranarray(x) for x in tend_inputs(p, dims, m.Np, m.NeA)]
    for f in fields:
        sdg.update_halo(f, m)
    g = gold[f"tend_{kind}_p{p}"]
    flags = sdg.FLAG_EXACT | (sdg.FLAG_ORDER_GENERAL if kind == "GENERAL" else 0)
    h = sdg.Handle(ops, m, flags)
    assert np.array_equal(h.cal_tend(*fields)[:, : m.Ne], g)
    h.close()
    h = sdg.Handle(ops, m, 0)
    assert rel_maxnorm(h.cal_tend(*fields)[:, : m.Ne], g) <= 1e-12
    h.close()


@pytest.mark.parametrize("name", sorted(MAIN_CASES))
def test_driver_matches_reference_program(name, tmp_path):
    run = os.path.join(sdg.PKG_DIR, "sdg_run")
    shutil.copytree(sdg.OPERATOR_DIR, tmp_path / "operator_data")
    (tmp_path / "input.conf").write_text(MAIN_CASES[name])
    r = subprocess.run([run, "input.conf"], capture_output=True, text=True,
                       cwd=tmp_path, timeout=300)
    assert r.returncode == 0, r.stderr
    got = [ln for ln in r.stdout.split("\n") if re.match(r"^\s*\d+\s+\S+\s+\S+$", ln)]
    assert got == main_lines()[name]
