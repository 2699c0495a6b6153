"""The C ABI (CPU only): the library loads, exports every entry point include/oos_gpu.h declares with the signature
the bindings give it, reports no device here without crashing, and its model helpers build matrices the reference
accepts. No compute call reaches a GPU."""

import os
import re

import numpy as np
import pytest

from conftest import has_gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "oos_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(oosgpu_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    from o_o_solver_b200 import _native

    names = declared_functions()
    assert len(names) >= 25
    bound = {name for name, _, _ in _native.SIGNATURES}
    for name in names:
        assert hasattr(lib, name), name
        assert name in bound, f"{name} has no binding"


def test_library_is_built_for_sm100a(lib):
    from o_o_solver_b200 import build

    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)
    assert os.path.exists(build.LIBRARY)


@pytest.mark.skipif(has_gpu(), reason="checks the behaviour without a device")
def test_no_device_is_an_error_not_a_fallback(lib, oracle_mod):
    from o_o_solver_b200 import SupernodalFactor, SymbolicFactor, device_count, linalg

    assert device_count() == 0
    symbolic = SymbolicFactor.from_arrays(2, [0, 2], [-1], [0, 0], [])
    with pytest.raises(linalg.CudaError):
        SupernodalFactor(symbolic)


def test_model_matrices_are_accepted_by_the_reference(lib, oracle_mod):
    """The stiffness and lumped mass in the reference's order: columns ascending from their diagonal, inside the
    symbolic structure (the reference factorises them; the mass has the stiffness's pattern)."""
    from o_o_solver_b200 import workloads

    model = workloads.Model(workloads.HexSpec(5))
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    k = model.csc(sym.node_order, 0)
    m = model.csc(sym.node_order, 1)
    assert np.array_equal(k.offsets, m.offsets) and np.array_equal(k.rows, m.rows)
    for j in range(k.dimension):
        col = k.rows[k.offsets[j]:k.offsets[j + 1]]
        assert col[0] == j and np.all(np.diff(col) > 0)
    f = oracle_mod.factorise(sym, k.offsets, k.rows, k.values)
    assert f.positive == sym.dof_count
    mass_diagonal = m.values[m.offsets[:-1]]
    assert np.all(mass_diagonal > 0)
    off = np.ones(len(m.values), bool)
    off[m.offsets[:-1]] = False
    assert np.all(m.values[off] == 0.0)
    # The lumped mass of the free nodes, 3 directions: the cube's mass but the half of its bottom layer that lumps
    # onto the clamped base.
    assert mass_diagonal.sum() == pytest.approx(3 * 7850.0 * (1.0 - 0.5 / 5.0), rel=1e-12)


def test_loads_are_seeded_and_placed(lib):
    from o_o_solver_b200 import workloads

    model = workloads.Model(workloads.PlateSpec(10, 10))
    order = np.arange(model.node_count, dtype=np.int32)
    a = model.loads(order, 5)
    b = model.loads(order, 5)
    assert np.array_equal(a, b)
    # pressure: p * area on the out-of-plane DOFs, summed over the free nodes (a clamped edge takes its share)
    assert a[2::6, 0].sum() == pytest.approx(1000.0 * 1.0 * (1.0 - 0.5 / 10), rel=1e-12)
    for j in range(1, 5):
        nonzero = np.nonzero(a[:, j])[0]
        assert 0 < len(nonzero) <= 10 and np.all(nonzero % 6 == 2)


def test_plate_model_sizes(lib):
    from o_o_solver_b200 import workloads

    model = workloads.Model(workloads.PlateSpec(100, 100))
    assert model.dof_count == 60600  # 101 x 101 grid points, the clamped edge removed, 6 DOFs each
    model = workloads.Model(workloads.HexSpec(10))
    assert model.dof_count == 11 * 11 * 10 * 3
