"""The partial factorisation of a unit (PartialFactor) against the reference's: the interior of a plate or a solid
factorised on the GPU with its boundary (the reference's trailing set, ordered last) left as the Schur complement K*,
the condensed loads f* = f_b - K_bi K_ii^-1 f_i and the recovery of the interior from boundary values, each within a
bound set by the spread between two of the reference's own kernel families; the recovery of K*'s own solution gives
the full solve of the unit."""

import numpy as np
import pytest

from conftest import has_gpu, relative_columns

pytestmark = pytest.mark.gpu

CASES = [("plate", 20), ("plate", 60), ("hex", 8), ("hex", 14)]


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def unit(kind, size, oracle):
    """A model with its boundary as the trailing set: the plate's free edge (x = lx), the solid's top face."""
    from o_o_solver_b200 import SymbolicFactor, workloads

    model = workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))
    axis = 0 if kind == "plate" else 2
    coordinate = model.coordinates[:, axis]
    boundary = np.flatnonzero(np.isclose(coordinate, coordinate.max())).astype(np.int32)
    sym = oracle.analyse(model.offsets, model.neighbours, model.weights, model.coordinates, trailing_nodes=boundary)
    assert sym.trailing_dofs == len(boundary) * model.node_dofs
    k = model.csc(sym.node_order, 0)
    symbolic = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    return model, sym, symbolic, k


def relative(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("kind,size", CASES, ids=[f"{k}{s}" for k, s in CASES])
def test_partial_factor_matches_reference(kind, size, lib, oracle_mod, gpu):
    from o_o_solver_b200 import FactorSolve, PartialFactor, SupernodalFactor

    model, sym, symbolic, k = unit(kind, size, oracle_mod)
    t = sym.trailing_dofs
    ref = oracle_mod.RefPartial(sym, k.offsets, k.rows, k.values, family=0)
    other = oracle_mod.RefPartial(sym, k.offsets, k.rows, k.values, family=1)
    partial = PartialFactor.factorise(symbolic, k, t)
    assert partial.inertia.positive == sym.dof_count - t and partial.inertia.negative == 0
    k_spread = relative(other.schur_complement, ref.schur_complement)
    k_difference = relative(partial.schur_complement, ref.schur_complement)
    assert np.array_equal(partial.schur_complement, partial.schur_complement.T)
    loads = model.loads(sym.node_order, 4)
    f_ref = ref.condense(loads)
    f_spread = relative(other.condense(loads), f_ref)
    f_difference = relative(partial.condense_loads(loads), f_ref)
    u_b = np.linalg.solve(ref.schur_complement, f_ref)
    u_ref = ref.recover(loads, u_b)
    u_spread = relative_columns(other.recover(loads, u_b), u_ref).max()
    u = partial.recover(loads, u_b)
    u_difference = relative_columns(u, u_ref).max()
    print(f"{kind}{size} ({t} boundary equations): K* {k_difference:.2e} (families {k_spread:.2e}), f* "
          f"{f_difference:.2e} ({f_spread:.2e}), recovery {u_difference:.2e} ({u_spread:.2e})")
    assert k_difference <= max(1e-13, 100.0 * k_spread)
    assert f_difference <= max(1e-13, 100.0 * f_spread)
    assert u_difference <= max(1e-12, 100.0 * u_spread)
    assert np.array_equal(u[sym.dof_count - t:], u_b)
    # K*'s own solution recovered: the unit's full solution
    full = SupernodalFactor.factorise(symbolic, k)
    x = np.array(loads, order="F", copy=True)
    FactorSolve(full).solve(x)
    own = partial.recover(loads, np.linalg.solve(partial.schur_complement, partial.condense_loads(loads)))
    assert relative_columns(own, x).max() <= 1e-8
    with pytest.raises(ValueError):  # a partial factor has no full solve
        FactorSolve(partial._factor).solve(np.array(loads, order="F", copy=True))
    full.close()
    partial.close()


def test_partial_factor_needs_a_trailing_set(lib, oracle_mod, gpu):
    """A symbolic factor whose last supernode is not the given trailing set is refused (std::invalid_argument)."""
    from o_o_solver_b200 import PartialFactor, SymbolicFactor, workloads

    model = workloads.Model(workloads.PlateSpec(10, 10))
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    k = model.csc(sym.node_order, 0)
    symbolic = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    last = int(sym.first_column[-1] - sym.first_column[-2])
    with pytest.raises(ValueError):
        PartialFactor.factorise(symbolic, k, last + 6)
