"""The statics benchmark's own workload against the reference: the 580 x 580 plate (2,021,880 equations, the
committed ordering the reference made), its 64 load cases (the pressure and 63 seeded patterns of point loads),
factorised and solved on the GPU and by the reference's own supernodal factorisation and solve on the host cores
(all of them, both kernel families): the same inertia and ratio-test figures, a backward error at FP64 rounding,
residuals within ten times the reference's, and the solutions within the bound the reference's two families set."""

import os

import numpy as np
import pytest

from conftest import has_gpu, relative_columns, solution_bound

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orderings")


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def test_plate580_statics_match_reference(lib, oracle_mod, gpu):
    from o_o_solver_b200 import FactorSolve, SupernodalFactor, SymbolicFactor, workloads

    threads = os.cpu_count() or 1
    fixture = np.load(os.path.join(GOLDEN, "plate580.npz"))
    order = fixture["node_order"]
    model = workloads.Model(workloads.PlateSpec(580, 580))
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, given_order=order, threads=threads)
    csc = model.csc(order)
    loads = model.loads(order, 64)
    symbolic = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, order,
                                             fixture["first_position"], fixture["parent"])
    assert symbolic.flop_count == sym.flops and symbolic.dof_count == sym.dof_count == 2021880
    factor = SupernodalFactor.factorise(symbolic, csc)
    x = np.asfortranarray(loads.copy())
    FactorSolve(factor).solve(x)
    solutions, ratios, equations = [], [], []
    for family in (1, 0):
        ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=family, threads=threads)
        assert (factor.inertia.positive, factor.inertia.negative, factor.inertia.zero) == (
            ref.positive, ref.negative, ref.zero)
        assert factor.pivot_diagnostics.issue_count == ref.issue_count
        ratios.append(ref.largest_ratio)
        equations.append(ref.equation_of_largest)
        solutions.append(ref.solve(loads, threads=threads))
        ref.close()
    # the largest a_jj / d_j: a drilling pivot of the thin plate, formed by cancellation, so its last digits differ
    # between any two correct factorisations; within ten times the reference families' own difference
    ratio_spread = abs(ratios[0] - ratios[1]) / abs(ratios[0])
    ratio_difference = abs(factor.pivot_diagnostics.largest_ratio - ratios[0]) / abs(ratios[0])
    assert ratio_difference <= max(1e-8, 10.0 * ratio_spread), (ratio_difference, ratio_spread)
    assert factor.pivot_diagnostics.equation_of_largest_ratio in equations
    factor.close()
    assert np.all(np.isfinite(x))
    r = loads - workloads.lower_csc_multiply(csc, x)
    absolute = workloads.SymmetricCsc(csc.offsets, csc.rows, np.abs(csc.values))
    norm_a = workloads.lower_csc_multiply(absolute, np.ones((csc.dimension, 1)))[:, 0].max()
    backward = np.abs(r).max(axis=0) / (norm_a * np.abs(x).max(axis=0) + np.abs(loads).max(axis=0))
    assert backward.max() <= 1e-15, backward.max()
    residual = relative_columns(workloads.lower_csc_multiply(csc, x), loads).max()
    reference_residual = relative_columns(workloads.lower_csc_multiply(csc, solutions[0]), loads).max()
    assert residual <= 10.0 * reference_residual + 1e-13, (residual, reference_residual)
    spread = relative_columns(solutions[1], solutions[0]).max()
    difference = relative_columns(x, solutions[0]).max()
    print(f"plate580, 64 columns: backward error {backward.max():.2e}, residual {residual:.2e} (reference "
          f"{reference_residual:.2e}), solution difference {difference:.2e} (reference families {spread:.2e}), "
          f"largest ratio difference {ratio_difference:.2e} (families {ratio_spread:.2e})")
    assert difference <= solution_bound(spread), (difference, spread)
