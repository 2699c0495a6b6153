"""The solves' chain launches as the host plans them (CPU only): per level with a large supernode (more than 64
columns), one forward and one backward launch; a task per 64-row block of each large supernode's x_F in both, and per
64 update rows in the forward one; a ready flag per block and direction. Building the plan checks that every task is
listed after the blocks it waits on, which the chains' progress rests on."""

import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orderings")


def expected_chains(first_column, parent, row_start):
    c = np.diff(np.asarray(first_column, dtype=np.int64))
    r = np.diff(np.asarray(row_start, dtype=np.int64))
    level = np.zeros(len(c), dtype=np.int64)
    for s, p in enumerate(parent):  # children before parents
        if p >= 0:
            level[p] = max(level[p], level[s] + 1)
    large = c > 64
    blocks = (c + 63) // 64
    rows = (r + 63) // 64
    forward = {}
    backward = {}
    for s in np.flatnonzero(large):
        forward[level[s]] = forward.get(level[s], 0) + blocks[s] + rows[s]
        backward[level[s]] = backward.get(level[s], 0) + blocks[s]
    return {"launches": 2 * len(forward), "tasks": int(sum(forward.values()) + sum(backward.values())),
            "flags": int(2 * blocks[large].sum()),
            "largest_launch": int(max(list(forward.values()) + list(backward.values()), default=0))}


@pytest.mark.parametrize("kind,size", [("plate", 20), ("plate", 40), ("hex", 8), ("hex", 12)])
def test_chain_launches_cover_the_large_supernodes(kind, size, oracle_mod, lib):
    from o_o_solver_b200 import SymbolicFactor, workloads

    model = workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    mine = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    chains = mine.solve_chains()
    assert chains == expected_chains(sym.first_column, sym.parent, sym.row_start)
    assert chains["launches"] > 0


@pytest.mark.parametrize("name", ["plate580", "hex60"])
def test_chain_launches_of_the_benchmark_workloads(name, lib):
    """The 2 M plate's and the 60^3 block's plans: the largest chain launch (the 60^3 block's root, 16,560 columns,
    259 blocks) and the flags the sweeps reset."""
    from o_o_solver_b200 import SymbolicFactor, workloads

    kind = "plate" if name.startswith("plate") else "hex"
    size = int(name[len(kind):])
    model = workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))
    fixture = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    mine = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, fixture["node_order"],
                                         fixture["first_position"], fixture["parent"])
    row_start, _ = mine.row_structure()
    weights = np.asarray(model.weights, dtype=np.int64)[fixture["node_order"]]
    column_of_position = np.concatenate([[0], np.cumsum(weights)])
    first_column = column_of_position[fixture["first_position"]]
    chains = mine.solve_chains()
    assert chains == expected_chains(first_column, fixture["parent"], row_start)
