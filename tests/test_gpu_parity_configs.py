"""Parity with the reference at the measured configurations, on the same symbolic factor and the same matrix:

- the 580 x 580 plate (2,021,880 equations) with its 64-column load block, the statics workload the benchmark
  times: the GPU factor and solve against the reference's own SupernodalFactor / FactorSolve (oracle/_ref);
- stiffened panels of the batched form: the joined GPU factorisation against each panel's own reference
  factorisation and solve.

Tolerances, stated per check:
- inertia, pivot diagnostics: exact;
- panels: within 1e-10 of the reference panel's largest magnitude (the top fronts of the plate, every supernode of the
  panels);
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

    ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, threads=THREADS)
    x_ref = ref.solve(b, threads=THREADS)
    # the largest fronts: the top of the tree, where the factorisation's long chains run
    sizes = np.diff(sym.first_column) * (np.diff(sym.first_column) + np.diff(sym.row_start))
    top = np.argsort(sizes)[-16:]
    ref_panels = {int(s): ref.panel(int(s)) for s in top}
    ref_inertia = (ref.positive, ref.negative, ref.zero)
    ref_diagnostics = (ref.issue_count, ref.equation_of_largest, ref.largest_ratio)
    ref.close()

    d_csc = SymmetricCsc(torch.from_numpy(csc.offsets).cuda(), torch.from_numpy(csc.rows).cuda(),
                         torch.from_numpy(csc.values).cuda())
    factor = SupernodalFactor.factorise(symbolic, d_csc)
    assert (factor.inertia.positive, factor.inertia.negative, factor.inertia.zero) == ref_inertia
    assert factor.pivot_diagnostics.issue_count == ref_diagnostics[0]
    assert factor.pivot_diagnostics.equation_of_largest_ratio == ref_diagnostics[1]
    assert factor.pivot_diagnostics.largest_ratio == pytest.approx(ref_diagnostics[2], rel=1e-8)
    worst_panel = 0.0
    for s, (theirs, ref_rows, _) in ref_panels.items():
        mine, rows, _ = factor.panel(s)
        assert np.array_equal(rows, ref_rows)
        worst_panel = max(worst_panel, np.abs(mine - theirs).max() / max(np.abs(theirs).max(), 1e-300))
    assert worst_panel <= 1e-10, worst_panel

    x = np.asfortranarray(b.copy())
    FactorSolve(factor).solve(x)
    factor.close()
    eta = backward_error(csc, x, b).max()
    difference = relative_columns(x, x_ref).max()
    # the reference's own spread on this matrix: its scalar kernel family against its automatic (SIMD) one
    scalar = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0, threads=THREADS)
    spread = relative_columns(scalar.solve(b, threads=THREADS), x_ref).max()
    print(f"plate580: panels {worst_panel:.2e}, backward error {eta:.2e}, solution difference {difference:.2e} "
          f"(reference families differ by {spread:.2e})")
    assert eta <= 1e-15, eta
    assert difference <= solution_bound(spread), (difference, spread)


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
