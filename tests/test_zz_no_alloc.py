"""The solve that allocates no device memory (oosgpu_solve_device_noalloc), for callers that cannot call cudaMalloc
once they are running (a fixed device-memory budget handed over at set-up). It is checked through the C ABI against
the ordinary device solve (oosgpu_solve_device) on the same factor, on two calls in a row (the second one reuses the
fixed scratch the first one left behind): for positive definite factors and for a pivoted indefinite one, with the
first call on a fresh factor made before any ordinary solve, and the device's free memory unchanged across the later
call. A factor too large for its fixed scratch is refused.

This file runs last (pytest collects it after the others): it passes alone in a fresh process and after the rest.
"""

import ctypes
import os

import numpy as np
import pytest

from conftest import has_gpu, relative_columns

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orderings")
# The tests' tolerance for two solves of one factor (the same kernels, narrower column tiles).
TOLERANCE = 1.0e-12


def factor_of(name, size, kind):
    from o_o_solver_b200 import SupernodalFactor, SymbolicFactor, workloads

    fixture = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    spec = workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size)
    model = workloads.Model(spec)
    symbolic = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, fixture["node_order"],
                                             fixture["first_position"], fixture["parent"])
    return model, fixture, symbolic, SupernodalFactor(symbolic)


@pytest.fixture(scope="module")
def torch_cuda():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def compare_solves(lib, torch, factor, n, columns, calls=2, seed=11):
    """`calls` rounds of: the solve without allocation, then the ordinary device solve, on the same right-hand
    sides. The first round's no-allocation call comes before any ordinary solve of the factor (so it cannot lean on
    buffers an ordinary solve would have left); from the second round on, the device's free memory is read around
    the no-allocation call and must not change."""
    rng = np.random.default_rng(seed)
    for call in range(calls):
        b = rng.standard_normal((columns, n))  # rows of this array are the columns of B
        fixed = torch.from_numpy(b).cuda()
        ordinary = torch.from_numpy(b).cuda()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        status = lib.oosgpu_solve_device_noalloc(factor._handle, fixed.data_ptr(), n, columns)
        assert status == 0, lib.oosgpu_last_error().decode()
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call > 0:
            assert free_after == free_before, f"call {call}: {free_before - free_after} bytes taken"
        status = lib.oosgpu_solve_device(factor._handle, ordinary.data_ptr(), n, columns)
        assert status == 0, lib.oosgpu_last_error().decode()
        torch.cuda.synchronize()
        expected = ordinary.cpu().numpy().T
        got = fixed.cpu().numpy().T
        assert np.all(np.isfinite(got)), f"call {call}"
        assert relative_columns(got, expected).max() <= TOLERANCE, f"call {call}"


@pytest.mark.parametrize("name,size,kind,columns", [("plate20", 20, "plate", 7), ("hex8", 8, "hex", 70)])
def test_noalloc_solve_matches_device_solve(name, size, kind, columns, lib, torch_cuda):
    torch = torch_cuda
    model, fixture, symbolic, factor = factor_of(name, size, kind)
    factor.refactorise(model.csc(fixture["node_order"]))
    compare_solves(lib, torch, factor, symbolic.dof_count, columns)


def test_noalloc_solve_of_a_pivoted_factor(lib, torch_cuda):
    """An indefinite factor (K - sigma M of the 8^3 block between its roots, Bunch-Kaufman pivots): the solve in pivot
    order with its 2 x 2 blocks, through the fixed scratch. A zero-column call first: the set-up call a caller makes
    before its working phase."""
    torch = torch_cuda
    from o_o_solver_b200 import FactorOptions, SymmetricCsc

    model, fixture, symbolic, factor = factor_of("hex8", 8, "hex")
    k = model.csc(fixture["node_order"], 0)
    m = model.csc(fixture["node_order"], 1)
    factor.refactorise(SymmetricCsc(k.offsets, k.rows, k.values - 2.0e8 * m.values),
                       FactorOptions(pivoting="indefinite"))
    assert factor.inertia.negative > 0
    n = symbolic.dof_count
    empty = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert lib.oosgpu_solve_device_noalloc(factor._handle, empty.data_ptr(), n, 0) == 0, \
        lib.oosgpu_last_error().decode()
    compare_solves(lib, torch, factor, n, 9, seed=5)


def test_noalloc_solve_refuses_a_factor_beyond_its_scratch(lib, torch_cuda):
    torch = torch_cuda
    model, fixture, symbolic, factor = factor_of("plate580", 580, "plate")
    x = torch.zeros(symbolic.dof_count, dtype=torch.float64, device="cuda")
    status = lib.oosgpu_solve_device_noalloc(factor._handle, x.data_ptr(), symbolic.dof_count, 1)
    assert status == 1  # OOSGPU_INVALID_ARGUMENT
    assert "scratch" in lib.oosgpu_last_error().decode()
