"""The oracle pinned before it is trusted (CPU only).

- The reference library (oracle/_ref/liboos_ref.so) is the reference's own code built from its sources; it reproduces
  the committed golden answers it made (tests/golden/solutions) and the known answers of the reference's checks
  (checks/linalg/FactorEdgeChecks.cpp:51-104, a chain of equations; a diagonal matrix).
- The C restatement (oracle/ldlt_port.c) gives the reference family's factor bit for bit (the same chains, no fused
  products) on plates and solids, and its solves agree to rounding.
"""

import os

import numpy as np
import pytest

from conftest import relative_columns

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def model_case(kind, size):
    from o_o_solver_b200 import workloads

    return workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))


def chain_graph(count):
    """A chain of `count` nodes of one DOF (node k adjacent to k - 1 and k + 1)."""
    offsets = [0]
    neighbours = []
    for k in range(count):
        if k > 0:
            neighbours.append(k - 1)
        if k + 1 < count:
            neighbours.append(k + 1)
        offsets.append(len(neighbours))
    return np.array(offsets, dtype=np.int64), np.array(neighbours, dtype=np.int32), np.ones(count, dtype=np.int32)


def chain_matrix(order, diagonal=4.0, off=-1.0):
    """The lower CSC of a tridiagonal matrix on the chain, in the given node order."""
    n = len(order)
    position = np.empty(n, dtype=np.int64)
    position[order] = np.arange(n)
    columns = [[] for _ in range(n)]
    for node in range(n):
        p = position[node]
        columns[p].append((p, diagonal))
        for other in (node - 1, node + 1):
            if 0 <= other < n and position[other] > p:
                columns[p].append((position[other], off))
    offsets = [0]
    rows = []
    values = []
    for col in columns:
        col.sort()
        rows += [r for r, _ in col]
        values += [v for _, v in col]
        offsets.append(len(rows))
    return np.array(offsets, dtype=np.int64), np.array(rows, dtype=np.int32), np.array(values)


@pytest.mark.parametrize("name", ["plate6", "plate20", "hex4", "hex8"])
def test_reference_reproduces_golden(name, oracle_mod, lib):
    kind = "plate" if name.startswith("plate") else "hex"
    size = int(name[len(kind):])
    model = model_case(kind, size)
    fixture = np.load(os.path.join(GOLDEN, "orderings", f"{name}.npz"))
    known = np.load(os.path.join(GOLDEN, "solutions", f"{name}.npz"))
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    assert np.array_equal(sym.node_order, fixture["node_order"])
    assert np.array_equal(sym.first_position, fixture["first_position"])
    assert np.array_equal(sym.parent, fixture["parent"])
    csc = model.csc(sym.node_order)
    factor = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0)
    assert [factor.positive, factor.negative, factor.zero] == list(known["inertia"])
    assert factor.issue_count == int(known["issue_count"])
    assert np.array_equal(factor.solve(known["b"]), known["x"])


@pytest.mark.parametrize("name", ["plate6", "plate20", "hex4", "hex8"])
def test_port_is_bit_exact_with_reference_family(name, oracle_mod, lib):
    kind = "plate" if name.startswith("plate") else "hex"
    size = int(name[len(kind):])
    model = model_case(kind, size)
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    csc = model.csc(sym.node_order)
    ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0)
    port = oracle_mod.PortFactor(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows, csc.offsets,
                                 csc.rows, csc.values)
    assert port.status == 0
    assert list(port.inertia) == [ref.positive, ref.negative, ref.zero]
    for s in range(sym.supernode_count):
        assert np.array_equal(port.panel(s), ref.panel(s)[0]), s
    b = np.asfortranarray(np.random.default_rng(1).standard_normal((sym.dof_count, 3)))
    assert relative_columns(port.solve(b), ref.solve(b)).max() < 1e-12


def test_port_reproduces_golden(oracle_mod, lib):
    model = model_case("plate", 6)
    fixture = np.load(os.path.join(GOLDEN, "orderings", "plate6.npz"))
    known = np.load(os.path.join(GOLDEN, "solutions", "plate6.npz"))
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, given_order=fixture["node_order"])
    csc = model.csc(sym.node_order)
    port = oracle_mod.PortFactor(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows, csc.offsets,
                                 csc.rows, csc.values)
    assert list(port.inertia) == list(known["inertia"])
    assert relative_columns(port.solve(known["b"]), known["x"]).max() < 1e-9


def test_chain_known_answer(oracle_mod):
    """A 3 000-equation tridiagonal chain and 3 right-hand sides (the shape of FactorEdgeChecks.cpp:191): the
    solution of [-1, 4, -1] x = b is checked by its residual, in the reference and the restatement."""
    offsets, neighbours, weights = chain_graph(3000)
    sym = oracle_mod.analyse(offsets, neighbours, weights, method=1)
    c_off, c_rows, c_vals = chain_matrix(sym.node_order)
    ref = oracle_mod.factorise(sym, c_off, c_rows, c_vals, family=0)
    assert (ref.positive, ref.negative, ref.zero) == (3000, 0, 0)
    port = oracle_mod.PortFactor(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows, c_off, c_rows,
                                 c_vals)
    b = np.asfortranarray(np.random.default_rng(2).standard_normal((3000, 3)))
    for x in (ref.solve(b), port.solve(b)):
        lower = np.zeros((3000, 3))
        # A x on the chain in factor order
        full = np.zeros((3000, 3000))
        for j in range(3000):
            for k in range(c_off[j], c_off[j + 1]):
                full[c_rows[k], j] = c_vals[k]
                full[j, c_rows[k]] = c_vals[k]
        lower = full @ x
        assert relative_columns(lower, b).max() < 1e-14


def test_diagonal_known_answer(oracle_mod):
    """A diagonal matrix (nodes without neighbours): D is the matrix, x = b / d, inertia from the signs."""
    n = 50
    offsets = np.zeros(n + 1, dtype=np.int64)
    neighbours = np.zeros(0, dtype=np.int32)
    weights = np.ones(n, dtype=np.int32)
    sym = oracle_mod.analyse(offsets, neighbours, weights, method=3)
    d = np.linspace(1.0, 5.0, n)
    c_off = np.arange(n + 1, dtype=np.int64)
    rows = np.arange(n, dtype=np.int32)
    values = d[sym.node_order]
    ref = oracle_mod.factorise(sym, c_off, rows, values, family=0)
    b = np.ones((n, 1))
    assert np.allclose(ref.solve(b)[:, 0], 1.0 / values, rtol=0, atol=1e-15)
    port = oracle_mod.PortFactor(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows, c_off, rows,
                                 values)
    assert np.array_equal(port.solve(b)[:, 0], 1.0 / values)


def test_port_zero_pivot_matches_reference(oracle_mod, lib):
    """A DOF without stiffness: the restatement's first zero pivot is the equation the reference's SingularityError
    names first."""
    import re

    model = model_case("plate", 6)
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    csc = model.csc(sym.node_order)
    target = 100
    cols = np.repeat(np.arange(sym.dof_count), np.diff(csc.offsets))
    values = csc.values.copy()
    values[(csc.rows == target) | (cols == target)] = 0.0
    with pytest.raises(RuntimeError) as raised:
        oracle_mod.factorise(sym, csc.offsets, csc.rows, values, family=0)
    named = [int(v) for v in re.findall(r"equation (\d+)", str(raised.value))]
    port = oracle_mod.PortFactor(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows, csc.offsets,
                                 csc.rows, values)
    assert port.status > 0
    assert port.zero_pivot_equation == min(named)
