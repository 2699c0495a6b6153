"""The symbolic structure the GPU path takes (CPU only): the row structures computed from the reference's node
order and supernode partition equal the reference's own (SymbolicFactor::analyse) bit for bit, on several graphs,
orderings and amalgamations; its counts equal the reference's; malformed structures are refused."""

import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orderings")


def model_case(kind, size):
    from o_o_solver_b200 import workloads

    return workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))


CASES = [("plate", 6, 0, True), ("plate", 20, 0, True), ("plate", 40, 0, True), ("plate", 12, 1, True),
         ("plate", 12, 3, False), ("hex", 4, 0, True), ("hex", 8, 0, True), ("hex", 12, 1, True),
         ("hex", 6, 2, False)]


@pytest.mark.parametrize("kind,size,method,amalgamate", CASES)
def test_row_structures_match_reference(kind, size, method, amalgamate, oracle_mod, lib):
    from o_o_solver_b200 import SymbolicFactor

    model = model_case(kind, size)
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, model.coordinates, method=method,
                             amalgamate=amalgamate)
    mine = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, sym.node_order,
                                         sym.first_position, sym.parent)
    row_start, rows = mine.row_structure()
    assert np.array_equal(row_start, sym.row_start)
    assert np.array_equal(rows, sym.rows)
    assert mine.dof_count == sym.dof_count
    assert mine.supernode_count == sym.supernode_count
    assert mine.flop_count == sym.flops
    assert mine.panel_value_count == sym.panel_values
    assert mine.factor_entry_count == sym.factor_entries


def test_from_arrays_matches_from_partition(oracle_mod, lib):
    from o_o_solver_b200 import SymbolicFactor

    model = model_case("hex", 8)
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    a = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    b = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, sym.node_order,
                                      sym.first_position, sym.parent)
    assert (a.flop_count, a.level_count, a.update_value_count) == (b.flop_count, b.level_count, b.update_value_count)


@pytest.mark.parametrize("name", ["plate100", "plate580", "hex30", "hex60"])
def test_golden_orderings_give_the_reference_counts(name, lib):
    """The committed orderings of the benchmark workloads: the structure built from them has the reference's flop
    count (recorded with the fixture)."""
    from o_o_solver_b200 import SymbolicFactor

    kind = "plate" if name.startswith("plate") else "hex"
    model = model_case(kind, int(name[len(kind):]))
    fixture = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    mine = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, fixture["node_order"],
                                         fixture["first_position"], fixture["parent"])
    assert mine.dof_count == int(fixture["dof_count"])
    assert mine.supernode_count == int(fixture["supernode_count"])
    assert mine.flop_count == float(fixture["flops"])


def test_malformed_structures_are_refused(lib):
    from o_o_solver_b200 import SymbolicFactor

    good = dict(dof_count=4, first_column=[0, 2, 4], parent=[1, -1], row_start=[0, 2, 2], rows=[2, 3])
    SymbolicFactor.from_arrays(**good)
    bad_cases = [
        dict(good, parent=[0, -1]),              # a parent before its child
        dict(good, rows=[3, 2]),                 # rows not ascending
        dict(good, rows=[1, 3]),                 # a row among the supernode's own columns
        dict(good, first_column=[0, 2, 5]),      # columns beyond the DOF count
        dict(good, row_start=[0, 2, 3], rows=[2, 3, 3]),  # a root with rows below it
    ]
    for case in bad_cases:
        with pytest.raises(ValueError):
            SymbolicFactor.from_arrays(**case)


def test_child_rows_outside_parent_are_refused(lib):
    from o_o_solver_b200 import SymbolicFactor

    # Supernode 0 has row 5, which supernode 1 (its parent: columns 2-3, rows 4) does not hold.
    with pytest.raises(ValueError):
        SymbolicFactor.from_arrays(6, [0, 2, 4, 6], [1, 2, -1], [0, 1, 2, 2], [5, 4])
