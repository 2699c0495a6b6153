"""The shifted pencil on the GPU (SparsePencil, include/oos/linalg/eigen/SparsePencil.hpp:29-85) against the
reference: the Sturm count of each shift is the reference's inertia of the same scaled shifted matrix, a solve applies
(K - shift M)^-1 to within FP64 backward error, the products with a lumped and with a coupled mass are M X, and the
properties the eigenvalue solver reads (the diagonal Rayleigh bound, the lumped flag, the factorisation count) are the
reference's definitions. Refusals: a negative mass diagonal (SolverError), two structures (ValueError)."""

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def hex_pencil(size, oracle):
    from o_o_solver_b200 import SymbolicFactor, workloads

    model = workloads.Model(workloads.HexSpec(size))
    sym = oracle.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    k = model.csc(sym.node_order, 0)
    m = model.csc(sym.node_order, 1)
    symbolic = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    return sym, symbolic, k, m


def scaled_shifted(k, m, sigma, scale):
    from o_o_solver_b200 import SymmetricCsc

    cols = np.repeat(np.arange(k.dimension), np.diff(k.offsets))
    return SymmetricCsc(k.offsets, k.rows, (k.values - sigma * m.values) * scale[k.rows] * scale[cols])


def test_sturm_counts_and_solves(lib, oracle_mod, gpu):
    from o_o_solver_b200 import SparsePencil, SymmetricCsc, workloads

    sym, symbolic, k, m = hex_pencil(10, oracle_mod)
    pencil = SparsePencil(symbolic, k, m)
    scale = oracle_mod.pencil_scale(k.offsets, k.rows, k.values)
    rng = np.random.default_rng(3)
    b = np.asfortranarray(rng.standard_normal((sym.dof_count, 4)))
    for count, sigma in enumerate([-1.0e6, 3.0e7, 2.5e8, 6.0e8], start=1):
        shift = pencil.factorise(sigma)
        s = scaled_shifted(k, m, sigma, scale)
        ref = oracle_mod.factorise(sym, s.offsets, s.rows, s.values, indefinite=True, family=0)
        assert shift.shift == sigma
        assert (shift.inertia.positive, shift.inertia.negative, shift.inertia.zero) == (ref.positive, ref.negative,
                                                                                        ref.zero)
        assert shift.sturm_count == ref.negative and not shift.is_singular
        assert pencil.factorisation_count == count
        x = pencil.solve(b.copy(order="F"))
        a = SymmetricCsc(k.offsets, k.rows, k.values - sigma * m.values)
        r = b - workloads.lower_csc_multiply(a, x)
        absolute = SymmetricCsc(a.offsets, a.rows, np.abs(a.values))
        norm_a = workloads.lower_csc_multiply(absolute, np.ones((a.dimension, 1)))[:, 0].max()
        eta = np.abs(r).max(axis=0) / (norm_a * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
        assert eta.max() <= 1e-14, sigma


def test_device_blocks_with_a_leading_dimension(lib, oracle_mod, gpu):
    """Device blocks whose columns are apart by more than the rows: only the rows of each column change."""
    from o_o_solver_b200 import SparsePencil

    torch = gpu
    sym, symbolic, k, m = hex_pencil(6, oracle_mod)
    pencil = SparsePencil(symbolic, k, m)
    pencil.factorise(1.0e8)
    n = sym.dof_count
    rng = np.random.default_rng(5)
    b = np.asfortranarray(rng.standard_normal((n, 3)))
    expected = pencil.solve(b.copy(order="F"))
    storage = torch.full((3, n + 7), 7.0, dtype=torch.float64, device="cuda")
    block = storage.t()[:n]
    block.copy_(torch.from_numpy(b))
    pencil.solve(block)
    torch.cuda.synchronize()
    assert np.array_equal(block.cpu().numpy(), expected)
    assert torch.all(storage[:, n:] == 7.0)
    y = torch.full((3, n + 5), 9.0, dtype=torch.float64, device="cuda").t()
    pencil.multiply_mass(block, y[:n])
    torch.cuda.synchronize()
    assert torch.all(y[n:] == 9.0)


def test_mass_products_lumped_and_coupled(lib, oracle_mod, gpu):
    from o_o_solver_b200 import SparsePencil, SymmetricCsc, workloads

    sym, symbolic, k, m = hex_pencil(7, oracle_mod)
    rng = np.random.default_rng(11)
    x = np.asfortranarray(rng.standard_normal((sym.dof_count, 37)))
    lumped = SparsePencil(symbolic, k, m)
    assert lumped.has_diagonal_mass
    y = lumped.multiply_mass(x, np.zeros_like(x, order="F"))
    assert np.array_equal(y, workloads.lower_csc_multiply(m, x))
    # A coupled mass on the whole pattern: |K| scaled (symmetric, positive diagonal).
    coupled = SymmetricCsc(k.offsets, k.rows, np.abs(k.values) * 1.0e-9)
    pencil = SparsePencil(symbolic, k, coupled)
    assert not pencil.has_diagonal_mass
    y = pencil.multiply_mass(x, np.zeros_like(x, order="F"))
    expected = workloads.lower_csc_multiply(coupled, x)
    assert np.abs(y - expected).max() <= 1e-13 * np.abs(expected).max()


def test_diagonal_rayleigh_bound(lib, oracle_mod, gpu):
    """min K_ii / M_ii over the equations with both positive (ShiftedPencil.hpp:80-85)."""
    from o_o_solver_b200 import SparsePencil, SymmetricCsc

    sym, symbolic, k, m = hex_pencil(5, oracle_mod)
    diag_k = k.values[k.offsets[:-1]]
    diag_m = m.values[m.offsets[:-1]].copy()
    diag_m[::4] = 0.0  # equations without mass do not bound
    values = m.values.copy()
    values[m.offsets[:-1]] = diag_m
    pencil = SparsePencil(symbolic, k, SymmetricCsc(m.offsets, m.rows, values))
    keep = (diag_m > 0) & (diag_k > 0)
    assert pencil.diagonal_rayleigh_bound == np.min(diag_k[keep] / diag_m[keep])
    massless = SparsePencil(symbolic, k, SymmetricCsc(m.offsets, m.rows, np.zeros_like(m.values)))
    assert massless.diagonal_rayleigh_bound == np.inf


def test_refusals(lib, oracle_mod, gpu):
    from o_o_solver_b200 import SolverError, SparsePencil, SymmetricCsc

    sym, symbolic, k, m = hex_pencil(4, oracle_mod)
    values = m.values.copy()
    values[m.offsets[3]] = -1.0
    with pytest.raises(SolverError, match="positive semi-definite"):
        SparsePencil(symbolic, k, SymmetricCsc(m.offsets, m.rows, values))
    rows = k.rows.copy()
    with pytest.raises(ValueError):
        SparsePencil(symbolic, k, SymmetricCsc(m.offsets[:-1], rows[:-1], m.values[:-1]))
