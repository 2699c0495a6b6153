"""The mixed-precision form of the factorisation (the update matrices of the large fronts by 3xTF32 products on the
tcgen05 tensor cores, FP32 accumulation): the inertia is the FP64 factor's, an unrefined solve is FP32-accurate (and no
better: the tensor-core path ran), and the FP64 iterative refinement of the solves recovers a backward error below
1e-13 on the solid blocks."""

import os

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orderings")


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def setup(kind, size):
    from o_o_solver_b200 import SymbolicFactor, workloads

    fx = np.load(os.path.join(GOLDEN, f"{kind}{size}.npz"))
    model = workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))
    symbolic = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, fx["node_order"],
                                             fx["first_position"], fx["parent"])
    return model, fx["node_order"], symbolic, model.csc(fx["node_order"], 0)


@pytest.mark.parametrize("size", [14, 30])
def test_mixed_factor_refines_to_fp64(size, lib, gpu):
    from o_o_solver_b200 import FactorOptions, SupernodalFactor, linalg

    torch = gpu
    model, order, symbolic, k = setup("hex", size)
    fp64 = SupernodalFactor.factorise(symbolic, k)
    mixed = SupernodalFactor.factorise(symbolic, k, FactorOptions(precision="mixed"))
    assert (mixed.inertia.positive, mixed.inertia.negative, mixed.inertia.zero) == (
        fp64.inertia.positive, fp64.inertia.negative, fp64.inertia.zero)
    dev = torch.device("cuda")
    b = torch.from_numpy(np.ascontiguousarray(model.loads(order, 8).T)).to(dev)
    x = torch.empty_like(b)
    unrefined = linalg.solve_refined(mixed, b.t(), x.t(), tolerance=1e-13, max_steps=0)
    assert 1e-12 < unrefined.backward_error < 1e-5, unrefined
    refined = linalg.solve_refined(mixed, b.t(), x.t(), tolerance=1e-13, max_steps=5)
    assert refined.backward_error <= 1e-13 and 1 <= refined.steps <= 5, refined
    exact = torch.empty_like(b)
    linalg.solve_refined(fp64, b.t(), exact.t(), tolerance=1e-15, max_steps=0)
    # the hexahedral block's first load column is zero (no pressure): its solution is zero in both forms
    difference = (x - exact).norm(dim=1) / exact.norm(dim=1).clamp_min(1e-300)
    assert float(difference.max()) <= 1e-9


def test_precision_is_checked(lib, gpu):
    from o_o_solver_b200 import FactorOptions, SupernodalFactor

    model, order, symbolic, k = setup("hex", 4)
    with pytest.raises(ValueError, match="precision"):
        SupernodalFactor.factorise(symbolic, k, FactorOptions(precision="fp16"))


def test_gmres_refinement_recovers_the_plate(lib, gpu):
    """The thin plate (60,600 equations) defeats classical refinement of the mixed factor (its conditioning times
    FP32's rounding is near 1); GMRES-IR with 12 Krylov vectors per correction reaches a backward error of 1e-10."""
    from o_o_solver_b200 import FactorOptions, SupernodalFactor, linalg

    torch = gpu
    model, order, symbolic, k = setup("plate", 100)
    mixed = SupernodalFactor.factorise(symbolic, k, FactorOptions(precision="mixed"))
    dev = torch.device("cuda")
    b = torch.from_numpy(np.ascontiguousarray(model.loads(order, 8).T)).to(dev)
    x = torch.empty_like(b)
    classical = linalg.solve_refined(mixed, b.t(), x.t(), tolerance=1e-10, max_steps=3)
    assert classical.backward_error > 1e-10
    gmres = linalg.solve_refined(mixed, b.t(), x.t(), tolerance=1e-10, max_steps=3, krylov=12)
    assert gmres.backward_error <= 1e-10, gmres
    with pytest.raises(ValueError, match="Krylov"):
        linalg.solve_refined(mixed, b.t(), x.t(), tolerance=1e-10, max_steps=3, krylov=13)
