"""Delayed pivots of the indefinite factorisation against the reference's (MultifrontalDriver::eliminatePivoted): on
matrices built so that Bunch-Kaufman must delay (the stiffness of plates and solids with the diagonal blocks of some
leaf supernodes scaled by 1e-6, so that each of their candidates has its column maximum outside the candidates and a
diagonal below 0.01 of it), the GPU delays the same candidates to the same parents: the same delayed-pivot count,
the same eliminated columns per supernode, the same inertia, and solves that are backward stable and agree with the
reference's. Where the GPU runs the reference's own algorithm throughout a subtree (small fronts, and the exact path
of the fronts that delay or grow), the panels themselves: rows in the reference's pivot order and values within
1e-10."""

import numpy as np
import pytest

from conftest import has_gpu, relative_columns

pytestmark = pytest.mark.gpu

# (kind, size, every k-th leaf supernode weakened)
CASES = [
    ("plate", 20, 7),
    ("hex", 8, 5),
    ("plate", 40, 11),
    ("hex", 14, 9),
]
SMALL_ORDER = 128  # fronts up to this order run the exact Bunch-Kaufman in shared memory


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def weakened(kind, size, every, oracle):
    """The stiffness with the diagonal blocks of every `every`-th leaf supernode scaled by 1e-6."""
    from o_o_solver_b200 import workloads

    model = workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))
    sym = oracle.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    k = model.csc(sym.node_order, 0)
    first = np.asarray(sym.first_column)
    parent = np.asarray(sym.parent)
    has_child = np.zeros(len(parent), dtype=bool)
    has_child[parent[parent >= 0]] = True
    chosen = [s for s in range(len(parent)) if not has_child[s]][::every]
    weak = np.zeros(k.dimension, dtype=bool)
    for s in chosen:
        weak[first[s]:first[s + 1]] = True
    cols = np.repeat(np.arange(k.dimension), np.diff(k.offsets))
    same = np.searchsorted(first, k.rows, side="right") == np.searchsorted(first, cols, side="right")
    values = k.values.copy()
    values[weak[k.rows] & weak[cols] & same] *= 1.0e-6
    return sym, workloads.SymmetricCsc(k.offsets, k.rows, values)


def backward_error(csc, x, b):
    from o_o_solver_b200 import workloads

    r = b - workloads.lower_csc_multiply(csc, x)
    absolute = workloads.SymmetricCsc(csc.offsets, csc.rows, np.abs(csc.values))
    norm_a = workloads.lower_csc_multiply(absolute, np.ones((csc.dimension, 1)))[:, 0].max()
    return np.abs(r).max(axis=0) / (norm_a * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))


def exact_subtrees(sym, ref):
    """The supernodes whose whole subtree the GPU factorises by the reference's own algorithm: fronts of order up to
    SMALL_ORDER, and fronts that delay or receive delayed columns (the exact path); the others take the block path,
    whose pivots may differ from the reference's."""
    parent = np.asarray(sym.parent)
    first = np.asarray(sym.first_column)
    row_start = np.asarray(sym.row_start)
    exact = np.zeros(len(parent), dtype=bool)
    for s in range(len(parent)):  # children before parents
        values, _, _ = ref.panel(s)
        order, eliminated = values.shape
        c = first[s + 1] - first[s]
        static = order == c + row_start[s + 1] - row_start[s] and eliminated == c
        exact[s] = order <= SMALL_ORDER or not static
    for s in range(len(parent)):
        if parent[s] >= 0 and not exact[s]:
            exact[parent[s]] = False
    return exact


@pytest.mark.parametrize("kind,size,every", CASES, ids=[f"{k}{s}" for k, s, _ in CASES])
def test_delays_match_reference(kind, size, every, lib, oracle_mod, gpu):
    from o_o_solver_b200 import FactorOptions, FactorSolve, SupernodalFactor, SymbolicFactor

    sym, a = weakened(kind, size, every, oracle_mod)
    # the reference family: the unblocked Bunch-Kaufman the exact path and the small fronts restate
    ref = oracle_mod.factorise(sym, a.offsets, a.rows, a.values, indefinite=True, family=0)
    assert ref.delayed > 0  # the matrix does make the reference delay
    symbolic = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    factor = SupernodalFactor.factorise(symbolic, a, FactorOptions(pivoting="indefinite"))
    print(f"{kind}{size}: delayed {factor.delayed_pivot_count} (reference {ref.delayed}), inertia "
          f"{factor.inertia} (reference {ref.positive}, {ref.negative}, {ref.zero})")
    assert factor.delayed_pivot_count == ref.delayed
    assert (factor.inertia.positive, factor.inertia.negative, factor.inertia.zero) == (ref.positive, ref.negative,
                                                                                       ref.zero)
    worst = 0.0
    exact = exact_subtrees(sym, ref)
    print(f"   {int(exact.sum())} of {len(exact)} supernodes on the reference's own algorithm throughout their subtree")
    for s in range(len(sym.parent)):
        mine, my_rows, my_sub = factor.panel(s)
        theirs, their_rows, their_sub = ref.panel(s)
        assert mine.shape == theirs.shape, s  # the same eliminated columns over the same grown front
        e = theirs.shape[1]
        assert set(my_rows[:e].tolist()) == set(their_rows[:e].tolist()), s
        assert set(my_rows.tolist()) == set(their_rows.tolist()), s
        if exact[s]:
            if not np.array_equal(my_rows, their_rows):
                at = int(np.flatnonzero(my_rows != their_rows)[0])
                raise AssertionError(f"supernode {s} (eliminated {e}): row {at} differs: "
                                     f"{my_rows[max(at - 3, 0):at + 6].tolist()} vs "
                                     f"{their_rows[max(at - 3, 0):at + 6].tolist()}")
            if e:
                worst = max(worst, np.abs(mine - theirs).max() / max(np.abs(theirs).max(), 1e-300))
                assert np.allclose(my_sub, their_sub, rtol=1e-10, atol=0.0), s
    assert worst <= 1e-10, worst
    rng = np.random.default_rng(size)
    b = np.asfortranarray(rng.standard_normal((sym.dof_count, 5)))
    x = b.copy(order="F")
    FactorSolve(factor).solve(x)
    assert np.all(np.isfinite(x))
    error = backward_error(a, x, b).max()
    x_ref = ref.solve(b)
    spread = relative_columns(
        oracle_mod.factorise(sym, a.offsets, a.rows, a.values, indefinite=True, family=1).solve(b), x_ref).max()
    difference = relative_columns(x, x_ref).max()
    print(f"   backward error {error:.2e}, difference {difference:.2e} (reference families {spread:.2e})")
    assert error <= 1e-13
    assert difference <= max(100.0 * spread, 1e-9)
    factor.close()


def test_delays_then_plain_refactorisation(lib, oracle_mod, gpu):
    """A factor that delayed, refactorised with a matrix that delays nothing: the solves go back to the plan's own
    structure (the restated one is dropped) and match the reference's."""
    from o_o_solver_b200 import FactorOptions, FactorSolve, SupernodalFactor, SymbolicFactor

    sym, a = weakened("hex", 8, 5, oracle_mod)
    from o_o_solver_b200 import workloads

    model = workloads.Model(workloads.HexSpec(8))
    k = model.csc(sym.node_order, 0)
    symbolic = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    options = FactorOptions(pivoting="indefinite")
    factor = SupernodalFactor.factorise(symbolic, a, options)
    assert factor.delayed_pivot_count > 0
    b = np.asfortranarray(np.random.default_rng(3).standard_normal((sym.dof_count, 3)))
    x = b.copy(order="F")
    FactorSolve(factor).solve(x)
    assert backward_error(a, x, b).max() <= 1e-13
    factor.refactorise(k, options)
    assert factor.delayed_pivot_count == 0
    assert (factor.inertia.positive, factor.inertia.negative) == (sym.dof_count, 0)
    y = b.copy(order="F")
    FactorSolve(factor).solve(y)
    assert backward_error(k, y, b).max() <= 1e-14
    factor.close()
