"""The solve that allocates no device memory (oosgpu_solve_device_noalloc), for callers that cannot call cudaMalloc
once they are running (a fixed device-memory budget handed over at set-up). It is checked through the C ABI against
the ordinary device solve (oosgpu_solve_device) on the same factor, on two calls in a row (the second one reuses the
fixed scratch the first one left behind), and a factor too large for its fixed scratch is refused.

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


@pytest.mark.parametrize("name,size,kind,columns", [("plate20", 20, "plate", 7), ("hex8", 8, "hex", 70)])
def test_noalloc_solve_matches_device_solve(name, size, kind, columns, lib, torch_cuda):
    torch = torch_cuda
    model, fixture, symbolic, factor = factor_of(name, size, kind)
    factor.refactorise(model.csc(fixture["node_order"]))
    n = symbolic.dof_count
    rng = np.random.default_rng(11)
    for call in range(2):
        b = rng.standard_normal((columns, n))  # rows of this array are the columns of B
        ordinary = torch.from_numpy(b).cuda()
        fixed = torch.from_numpy(b).cuda()
        torch.cuda.synchronize()
        status = lib.oosgpu_solve_device(factor._handle, ordinary.data_ptr(), n, columns)
        assert status == 0, lib.oosgpu_last_error().decode()
        status = lib.oosgpu_solve_device_noalloc(factor._handle, fixed.data_ptr(), n, columns)
        assert status == 0, lib.oosgpu_last_error().decode()
        torch.cuda.synchronize()
        expected = ordinary.cpu().numpy().T
        got = fixed.cpu().numpy().T
        assert np.all(np.isfinite(got)), f"call {call}"
        assert relative_columns(got, expected).max() <= TOLERANCE, f"call {call}"


def test_noalloc_solve_refuses_a_factor_beyond_its_scratch(lib, torch_cuda):
    torch = torch_cuda
    model, fixture, symbolic, factor = factor_of("plate580", 580, "plate")
    x = torch.zeros(symbolic.dof_count, dtype=torch.float64, device="cuda")
    status = lib.oosgpu_solve_device_noalloc(factor._handle, x.data_ptr(), symbolic.dof_count, 1)
    assert status == 1  # OOSGPU_INVALID_ARGUMENT
    assert "scratch" in lib.oosgpu_last_error().decode()
