"""Parity with the reference at the measured configurations, on the same symbolic factor and the same matrix:

- the 580 x 580 plate (2,021,880 equations) with its 64-column load block, the statics workload the benchmark
  times: the GPU factor and solve against the reference's own SupernodalFactor / FactorSolve (oracle/_ref);
- stiffened panels of the batched form: the joined GPU factorisation against each panel's own reference
  factorisation and solve.

Tolerances, stated per check:
- inertia, the count of ratio-test issues and the equation of the largest ratio: exact;
- panels: within 1e-10 of the reference panel's largest magnitude (every supernode of the panels); on the 2 M plate,
  whose top pivots are small against their diagonals (largest ratio about 3e5), within 100 x the distance between the
  reference's own two kernel families (scalar and SIMD) where that is larger, and so for the largest ratio (1e-8);
- backward error ||b - Ax||_inf / (||A||_inf ||x||_inf + ||b||_inf) of the GPU solution: at most 1e-15;
- solutions: relative 2-norm difference per column at most min(1e-9, 100 x spread) where the reference's own two
  kernel families agree to 1e-11 or better (spread = their difference). On the thin plates they do not: the 2 mm
  cantilever's conditioning makes two correct FP64 solves differ by about 1e-8 (200 x 200) or more, so there the
  bound is 100 x that spread. The achieved figures are printed.
"""

import os

import numpy as np
import pytest

from conftest import has_gpu, relative_columns, solution_bound

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orderings")
THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def backward_error(csc, x, b):
    from o_o_solver_b200 import workloads

    r = b - workloads.lower_csc_multiply(csc, x)
    absolute = workloads.SymmetricCsc(csc.offsets, csc.rows, np.abs(csc.values))
    norm_a = workloads.lower_csc_multiply(absolute, np.ones((csc.dimension, 1)))[:, 0].max()
    return np.abs(r).max(axis=0) / (norm_a * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))


def test_plate580_statics_matches_reference(lib, oracle_mod, gpu):
    """The benchmark's workload: factor + 64-column solve of the 2,021,880-equation plate."""
    torch = gpu
    from o_o_solver_b200 import FactorSolve, SupernodalFactor, SymbolicFactor, SymmetricCsc, workloads

    fixture = np.load(os.path.join(GOLDEN, "plate580.npz"))
    order = fixture["node_order"]
    model = workloads.Model(workloads.PlateSpec(580, 580))
    csc = model.csc(order)
    b = model.loads(order, 64)
    sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights, given_order=order, threads=THREADS)
    assert sym.dof_count == 2021880
    symbolic = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    assert symbolic.flop_count == pytest.approx(sym.flops, rel=1e-12)

    # the reference twice: its automatic (SIMD) kernel family, the comparison, and its scalar family, whose
    # distance from the first measures what two correct FP64 factorisations of this matrix can differ by
    sizes = np.diff(sym.first_column) * (np.diff(sym.first_column) + np.diff(sym.row_start))
    top = [int(s) for s in np.argsort(sizes)[-16:]]  # the largest fronts: the top of the tree
    runs = []
    for family in (-1, 0):
        ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=family, threads=THREADS)
        runs.append({"x": ref.solve(b, threads=THREADS), "panels": {s: ref.panel(s) for s in top},
                     "inertia": (ref.positive, ref.negative, ref.zero),
                     "diagnostics": (ref.issue_count, ref.equation_of_largest, ref.largest_ratio)})
        ref.close()
    ref, scalar = runs
    assert ref["inertia"] == scalar["inertia"]

    def panel_distance(panels):
        worst = 0.0
        for s, (theirs, ref_rows, _) in ref["panels"].items():
            mine, rows, _ = panels(s)
            assert np.array_equal(rows, ref_rows)
            worst = max(worst, np.abs(mine - theirs).max() / max(np.abs(theirs).max(), 1e-300))
        return worst

    panel_spread = panel_distance(lambda s: scalar["panels"][s])
    ratio_spread = abs(scalar["diagnostics"][2] - ref["diagnostics"][2]) / ref["diagnostics"][2]
    solution_spread = relative_columns(scalar["x"], ref["x"]).max()

    d_csc = SymmetricCsc(torch.from_numpy(csc.offsets).cuda(), torch.from_numpy(csc.rows).cuda(),
                         torch.from_numpy(csc.values).cuda())
    factor = SupernodalFactor.factorise(symbolic, d_csc)
    assert (factor.inertia.positive, factor.inertia.negative, factor.inertia.zero) == ref["inertia"]
    assert factor.pivot_diagnostics.issue_count == ref["diagnostics"][0]
    assert factor.pivot_diagnostics.equation_of_largest_ratio == ref["diagnostics"][1]
    ratio = abs(factor.pivot_diagnostics.largest_ratio - ref["diagnostics"][2]) / ref["diagnostics"][2]
    worst_panel = panel_distance(lambda s: factor.panel(s))
    x = np.asfortranarray(b.copy())
    FactorSolve(factor).solve(x)
    factor.close()
    eta = backward_error(csc, x, b).max()
    difference = relative_columns(x, ref["x"]).max()
    print(f"plate580 against the reference (its own two kernel families in brackets): top panels {worst_panel:.2e} "
          f"({panel_spread:.2e}), largest pivot ratio {ratio:.2e} ({ratio_spread:.2e}), solutions {difference:.2e} "
          f"({solution_spread:.2e}), GPU backward error {eta:.2e}")
    assert worst_panel <= max(1e-10, 100.0 * panel_spread), (worst_panel, panel_spread)
    assert ratio <= max(1e-8, 100.0 * ratio_spread), (ratio, ratio_spread)
    assert eta <= 1e-15, eta
    assert difference <= solution_bound(solution_spread), (difference, solution_spread)


PANEL_COUNT = 12


def test_panels_match_their_reference_factorisations(lib, oracle_mod, gpu):
    """The batched form: 12 seeded panels (the first of the benchmark's 512, mesh sizes drawn across the range)
    joined, factorised and solved on the GPU; each panel's supernodes and solution against the reference's
    factorisation and solve of that panel alone."""
    from o_o_solver_b200 import FactorSolve, SupernodalFactor, batch, workloads

    cases = batch.panel_cases(PANEL_COUNT)
    fixtures = {}

    def fixture_of(n):
        if n not in fixtures:
            fixtures[n] = dict(np.load(os.path.join(GOLDEN, f"panel{n}.npz")))
        return fixtures[n]

    joined, rhs, parts = batch.panel_batch(cases, fixture_of, columns=8)
    factor = SupernodalFactor.factorise(joined.symbolic, joined.matrix)
    x = np.asfortranarray(rhs.copy())
    FactorSolve(factor).solve(x)
    supernode = 0
    report = []
    for i, (case, part, xi, bi) in enumerate(zip(cases, parts, joined.split(x), joined.split(rhs))):
        model = workloads.Model(workloads.PanelSpec(n=case.n, stringers=case.stringers, thickness=case.thickness))
        sym = oracle_mod.analyse(model.offsets, model.neighbours, model.weights,
                                 given_order=fixture_of(case.n)["node_order"], threads=THREADS)
        model.close()
        assert np.array_equal(sym.first_column, part.first_column), i
        assert np.array_equal(sym.parent, part.parent), i
        ref = oracle_mod.factorise(sym, part.matrix.offsets, part.matrix.rows, part.matrix.values, threads=THREADS)
        assert (ref.negative, ref.zero) == (0, 0)
        worst_panel = 0.0
        offset = int(joined.dof_offsets[i])
        for s in range(sym.supernode_count):
            mine, rows, _ = factor.panel(supernode + s)
            theirs, ref_rows, _ = ref.panel(s)
            assert np.array_equal(rows, ref_rows + offset), (i, s)
            worst_panel = max(worst_panel, np.abs(mine - theirs).max() / max(np.abs(theirs).max(), 1e-300))
        supernode += sym.supernode_count
        x_ref = ref.solve(np.asfortranarray(bi), threads=THREADS)
        scalar = oracle_mod.factorise(sym, part.matrix.offsets, part.matrix.rows, part.matrix.values, family=0,
                                      threads=THREADS)
        spread = relative_columns(scalar.solve(np.asfortranarray(bi), threads=THREADS), x_ref).max()
        difference = relative_columns(xi, x_ref).max()
        eta = backward_error(part.matrix, xi, bi).max()
        report.append((case.n, case.stringers, worst_panel, difference, spread, eta))
        assert worst_panel <= 1e-10, (i, worst_panel)
        assert eta <= 1e-15, (i, eta)
        assert difference <= solution_bound(spread), (i, difference, spread)
    factor.close()
    for n, stringers, panel, difference, spread, eta in report:
        print(f"panel {n}x{n}, {stringers} blades: panels {panel:.1e}, solution {difference:.1e} "
              f"(reference families {spread:.1e}), backward error {eta:.1e}")
