"""The stiffness and lumped mass formed on the GPU (element matrices, node blocks, compressed columns) against the
host's: the same offsets, the same rows and the same values bit for bit, for every workload model family (plates,
solids, stiffened panels with frame blades, wing boxes with oriented shells), in the analysed order and in a shuffled
one. The host's columns are the reference's own assembly order (StiffnessAssembler, then SymmetricCsc::fromBlocks:
columns ascending from their diagonal)."""

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

CASES = [
    ("plate", 20),
    ("plate", 100),
    ("hex", 8),
    ("hex", 14),
    ("panel", 40),
    ("wing", 0),
]


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def build(kind, size):
    from o_o_solver_b200 import workloads

    if kind == "plate":
        return workloads.Model(workloads.PlateSpec(size, size))
    if kind == "hex":
        return workloads.Model(workloads.HexSpec(size))
    if kind == "panel":
        return workloads.Model(workloads.PanelSpec(size, 5))
    thicknesses = tuple(0.002 + 0.0002 * z for z in range(24))
    return workloads.Model(workloads.WingBoxSpec(thicknesses, span=2.0, h=0.1))


def same(host, device):
    assert np.array_equal(host.offsets, device.offsets.cpu().numpy())
    assert np.array_equal(host.rows, device.rows.cpu().numpy())
    got = device.values.cpu().numpy()
    assert got.shape == host.values.shape
    assert np.array_equal(host.values.view(np.int64), got.view(np.int64)), (
        f"{int(np.count_nonzero(host.values != got))} values differ")


@pytest.mark.parametrize("kind,size", CASES, ids=[f"{k}{s}" for k, s in CASES])
@pytest.mark.parametrize("ordering", ["analysed", "shuffled"])
def test_device_assembly_matches_host(gpu, oracle_mod, kind, size, ordering):
    model = build(kind, size)
    if ordering == "analysed":
        order = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, model.coordinates).node_order
    else:
        order = np.random.default_rng(size + 7).permutation(model.node_count).astype(np.int32)
    same(model.csc(order, 0), model.csc_device(order, 0))
    if kind in ("hex", "wing"):
        same(model.csc(order, 1), model.csc_device(order, 1))


def test_device_assembly_refuses_a_missing_mass(gpu):
    model = build("plate", 4)
    with pytest.raises(ValueError):
        model.csc_device(np.arange(model.node_count, dtype=np.int32), 1)
