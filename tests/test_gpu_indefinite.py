"""The indefinite factorisation on the GPU (PivotingMode::Indefinite) against the reference's own, on shifted and
scaled pencils S (K - sigma M) S of plates and solids: the inertia (the Sturm count of sigma: its negative pivots) is
exactly the reference's; the solves are backward stable and agree with the reference's solutions to within the
spread of two of the reference's own kernel families; a singular shifted matrix is counted, not refused, and refuses
its solves.

The GPU's pivots may differ from the reference's (Bunch-Kaufman inside each 64-column diagonal block with an
a-posteriori threshold test, the reference's exact algorithm for the small fronts and for any front the test refuses);
the inertia may not (Sylvester's law of inertia)."""

import numpy as np
import pytest

from conftest import has_gpu, relative_columns

pytestmark = pytest.mark.gpu

# (kind, size, shifts): shifts below, inside and above the lowest roots (the hex roots start near 1.2e7, the plate's
# near 105).
CASES = [
    ("hex", 8, [6.0e6, 2.0e8, 3.7e8]),
    ("hex", 14, [2.0e8, 3.7e8]),
    ("plate", 20, [50.0, 7.0e4, 1.7e5]),
    ("plate", 40, [7.0e4]),
]


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def pencil(kind, size, oracle):
    from o_o_solver_b200 import workloads

    model = workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))
    sym = oracle.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    k = model.csc(sym.node_order, 0)
    if kind == "hex":
        m = model.csc(sym.node_order, 1)
    else:  # a lumped mass on the translations of a 2 mm aluminium sheet
        values = np.zeros_like(k.values)
        mass = np.zeros(sym.dof_count)
        mass[np.arange(sym.dof_count) % 6 < 3] = 2700.0 * 0.002 / (size * size)
        values[k.offsets[:-1]] = mass
        m = workloads.SymmetricCsc(k.offsets, k.rows, values)
    return model, sym, k, m


def shifted(k, m, sigma, scale):
    from o_o_solver_b200 import SymmetricCsc

    cols = np.repeat(np.arange(k.dimension), np.diff(k.offsets))
    return SymmetricCsc(k.offsets, k.rows, (k.values - sigma * m.values) * scale[k.rows] * scale[cols])


def backward_error(csc, x, b):
    from o_o_solver_b200 import workloads

    r = b - workloads.lower_csc_multiply(csc, x)
    absolute = workloads.SymmetricCsc(csc.offsets, csc.rows, np.abs(csc.values))
    norm_a = workloads.lower_csc_multiply(absolute, np.ones((csc.dimension, 1)))[:, 0].max()
    return np.abs(r).max(axis=0) / (norm_a * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))


def gpu_factor(sym, matrix):
    from o_o_solver_b200 import FactorOptions, SupernodalFactor, SymbolicFactor

    symbolic = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    return SupernodalFactor.factorise(symbolic, matrix, FactorOptions(pivoting="indefinite"))


@pytest.mark.parametrize("kind,size,shifts", CASES)
def test_inertia_and_solves_match_reference(kind, size, shifts, lib, oracle_mod, gpu):
    from o_o_solver_b200 import FactorSolve

    model, sym, k, m = pencil(kind, size, oracle_mod)
    scale = oracle_mod.pencil_scale(k.offsets, k.rows, k.values)
    rng = np.random.default_rng(size)
    b = np.asfortranarray(rng.standard_normal((sym.dof_count, 5)))
    for sigma in shifts:
        a = shifted(k, m, sigma, scale)
        ref = oracle_mod.factorise(sym, a.offsets, a.rows, a.values, indefinite=True, family=0)
        factor = gpu_factor(sym, a)
        assert (factor.inertia.positive, factor.inertia.negative, factor.inertia.zero) == (
            ref.positive, ref.negative, ref.zero), sigma
        x = b.copy(order="F")
        FactorSolve(factor).solve(x)
        assert np.all(np.isfinite(x))
        x_ref = ref.solve(b)
        # backward stable: within the reference's own (2.1e-14 on the 14^3 block at 3.7e8, inside the spectrum)
        assert backward_error(a, x, b).max() <= max(1e-14, 2.0 * backward_error(a, x_ref, b).max()), sigma
        spread = relative_columns(
            oracle_mod.factorise(sym, a.offsets, a.rows, a.values, indefinite=True, family=1).solve(b), x_ref).max()
        assert relative_columns(x, x_ref).max() <= 100.0 * spread + 1e-11, sigma


def test_singular_shift_is_counted_and_refuses_solves(lib, oracle_mod, gpu):
    """A shifted matrix with a DOF that has neither stiffness nor mass: a zero pivot in the inertia (the reference
    counts it), and solving with the factor is refused (SingularityError)."""
    from o_o_solver_b200 import FactorSolve, SingularityError, SymmetricCsc

    model, sym, k, m = pencil("hex", 6, oracle_mod)
    target = sym.dof_count // 2
    cols = np.repeat(np.arange(sym.dof_count), np.diff(k.offsets))
    values = k.values - 2.0e8 * m.values
    values[(k.rows == target) | (cols == target)] = 0.0
    a = SymmetricCsc(k.offsets, k.rows, values)
    ref = oracle_mod.factorise(sym, a.offsets, a.rows, a.values, indefinite=True, family=0)
    assert ref.zero >= 1
    factor = gpu_factor(sym, a)
    assert (factor.inertia.positive, factor.inertia.negative, factor.inertia.zero) == (ref.positive, ref.negative,
                                                                                       ref.zero)
    with pytest.raises(SingularityError):
        FactorSolve(factor).solve(np.ones((sym.dof_count, 1), order="F"))


def test_positive_definite_matrix_in_indefinite_mode(lib, oracle_mod, gpu):
    """K itself factorised in indefinite mode: all pivots positive, the solution the positive definite mode's."""
    from o_o_solver_b200 import FactorSolve, SupernodalFactor, SymbolicFactor

    model, sym, k, m = pencil("plate", 20, oracle_mod)
    factor = gpu_factor(sym, k)
    assert (factor.inertia.positive, factor.inertia.negative, factor.inertia.zero) == (sym.dof_count, 0, 0)
    symbolic = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    pd = SupernodalFactor.factorise(symbolic, k)
    b = model.loads(sym.node_order, 3)
    x = b.copy(order="F")
    y = b.copy(order="F")
    FactorSolve(factor).solve(x)
    FactorSolve(pd).solve(y)
    assert backward_error(k, x, b).max() <= 1e-15
    spread = relative_columns(oracle_mod.factorise(sym, k.offsets, k.rows, k.values, family=1).solve(b),
                              oracle_mod.factorise(sym, k.offsets, k.rows, k.values, family=0).solve(b)).max()
    assert relative_columns(x, y).max() <= 100.0 * spread + 1e-12
