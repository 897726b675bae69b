"""The derivative operators on the GPU against the oracle.

sdg_divlike_dev replaces element_operation_kernel_matvec_divlike_dirXYZ_var5_P<p>
(mod_dg_optr_kernel_opt1.F90.erb:347-465) for any number of fields per
element; sdg_gradlike_dev replaces gradlike_dirXYZ_P<p> (erb:166-219).  Exact
mode must equal the oracle bit for bit in the OPT1 and GENERAL orders; the
FMA mode must agree to 1e-12 relative max-norm, the tolerance of the
tendency parity tests.
"""
import numpy as np
import pytest

import orc
import sdg_b200 as sdg
from conftest import rel_maxnorm

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


def _fields(p, nvar, Ne, seed, count=3):
    Np = (p + 1) ** 3
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(Ne * nvar * Np) for _ in range(count)]


def _run_div(ops, nvar, Ne, ins, flags):
    import torch

    dev = [torch.from_numpy(a).cuda() for a in ins]
    outs = [torch.full_like(dev[0], float("nan")) for _ in range(3)]
    sdg.divlike_dirXYZ_var_dev(ops.D1D, nvar, Ne, *dev, *outs, flags=flags)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs]


def _run_grad(ops, Ne, f, flags):
    import torch

    d = torch.from_numpy(f).cuda()
    outs = [torch.full_like(d, float("nan")) for _ in range(3)]
    sdg.gradlike_dirXYZ_dev(ops.D1D, Ne, d, *outs, flags=flags)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs]


@pytest.mark.parametrize("p", range(1, 16))
def test_divlike_var5_vs_oracle(p):
    """Five fields per element (the Euler-equation form), an element count
    that leaves a partial last block: exact OPT1 and GENERAL bit for bit,
    FMA within 1e-12."""
    ops = sdg.read_operators(p)
    nvar, Ne = 5, 7
    ins = _fields(p, nvar, Ne, seed=100 + p)
    for ev, flags in ((orc.OPT1, sdg.FLAG_EXACT),
                      (orc.GENERAL, sdg.FLAG_EXACT | sdg.FLAG_ORDER_GENERAL)):
        ref = orc.divlike_fields(ev, ops.D1D, nvar, Ne, *ins)
        got = _run_div(ops, nvar, Ne, ins, flags)
        for d in range(3):
            assert np.array_equal(got[d], ref[d]), (p, ev, d)
    ref = orc.divlike_fields(orc.OPT1, ops.D1D, nvar, Ne, *ins)
    got = _run_div(ops, nvar, Ne, ins, 0)
    for d in range(3):
        assert rel_maxnorm(got[d], ref[d]) <= TOL, (p, d)


@pytest.mark.parametrize("p", [1, 3, 5, 7, 9, 12, 15])
def test_gradlike_vs_oracle(p):
    ops = sdg.read_operators(p)
    Ne = 11
    (f,) = _fields(p, 1, Ne, seed=200 + p, count=1)
    ref = orc.divlike_fields(orc.OPT1, ops.D1D, 1, Ne, f, f, f)
    got = _run_grad(ops, Ne, f, sdg.FLAG_EXACT)
    for d in range(3):
        assert np.array_equal(got[d], ref[d]), (p, d)
    got = _run_grad(ops, Ne, f, 0)
    for d in range(3):
        assert rel_maxnorm(got[d], ref[d]) <= TOL, (p, d)


def test_divlike_one_field_and_empty():
    """nvar = 1 with three different inputs; Ne = 0 launches nothing."""
    import torch

    p = 7
    ops = sdg.read_operators(p)
    ins = _fields(p, 1, 3, seed=5)
    ref = orc.divlike_fields(orc.OPT1, ops.D1D, 1, 3, *ins)
    got = _run_div(ops, 1, 3, ins, sdg.FLAG_EXACT)
    for d in range(3):
        assert np.array_equal(got[d], ref[d])
    z = torch.zeros(1, dtype=torch.float64, device="cuda")
    sdg.divlike_dirXYZ_var_dev(ops.D1D, 5, 0, z, z, z, z, z, z)
    sdg.gradlike_dirXYZ_dev(ops.D1D, 0, z, z, z, z)
    torch.cuda.synchronize()


def test_gradlike_polynomial_exact():
    """Degree-p polynomials are differentiated exactly on the LGL nodes."""
    p = 6
    ops = sdg.read_operators(p)
    x = ops.x1D
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = (X ** 3 * Y ** 2 * Z).ravel(order="F")
    want = [(3 * X ** 2 * Y ** 2 * Z), (2 * X ** 3 * Y * Z), (X ** 3 * Y ** 2)]
    got = _run_grad(ops, 1, f, 0)
    for d in range(3):
        assert np.max(np.abs(got[d] - want[d].ravel(order="F"))) < 1e-11
