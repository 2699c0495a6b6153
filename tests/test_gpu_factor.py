"""Parity of the GPU factorisation and solves with the reference (oracle/_ref/liboos_ref.so, the reference's own
SupernodalFactor / FactorSolve built from its sources) on the same symbolic factor and the same matrix.

Tolerances: the inertia, the zero pivots and the ratio-test counts are exact; the panels agree to 1e-10 of their
norm; a solution's residual is within a small multiple of the reference's own; the solutions differ from the
reference's by at most min(1e-9, 100 x spread + 1e-12), spread being the difference between two of the reference's
own kernel families (scalar vs AVX2, on the same input), where that spread is 1e-11 or less (the solid blocks). The
thin plates are ill conditioned (the reference's residual is about 1e-7 on the 60 600 equations of the 100 x 100
plate), so two correct FP64 factors do not agree to more digits than their conditioning allows: there the bound is
100 x the spread (conftest.solution_bound).
"""

import numpy as np
import pytest

from conftest import has_gpu, relative_columns, solution_bound

pytestmark = pytest.mark.gpu

CASES = {
    "plate6": ("plate", 6),
    "plate20": ("plate", 20),
    "hex4": ("hex", 4),
    "hex8": ("hex", 8),
    "hex14": ("hex", 14),
    "plate100": ("plate", 100),
}


def build_case(name, oracle):
    from o_o_solver_b200 import workloads

    kind, size = CASES[name]
    spec = workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size)
    model = workloads.Model(spec)
    sym = oracle.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    csc = model.csc(sym.node_order)
    return model, sym, csc


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def gpu_symbolic(sym):
    from o_o_solver_b200 import SymbolicFactor

    return SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)


def residual(csc, x, b):
    """||b - A x|| / ||b|| per column."""
    from o_o_solver_b200 import workloads

    return relative_columns(workloads.lower_csc_multiply(csc, x), b)


def backward_error(csc, x, b):
    """The normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) per column (Rigal-Gaches)."""
    from o_o_solver_b200 import workloads

    r = b - workloads.lower_csc_multiply(csc, x)
    absolute = workloads.SymmetricCsc(csc.offsets, csc.rows, np.abs(csc.values))
    norm_a = workloads.lower_csc_multiply(absolute, np.ones((csc.dimension, 1)))[:, 0].max()
    if r.ndim == 1:
        r, x, b = r[:, None], x[:, None], b[:, None]
    return np.abs(r).max(axis=0) / (norm_a * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))


@pytest.mark.parametrize("name", list(CASES))
def test_factor_matches_reference(name, lib, oracle_mod, gpu):
    from o_o_solver_b200 import FactorSolve, SupernodalFactor

    model, sym, csc = build_case(name, oracle_mod)
    ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0)
    factor = SupernodalFactor.factorise(gpu_symbolic(sym), csc)
    assert (factor.inertia.positive, factor.inertia.negative, factor.inertia.zero) == (ref.positive, ref.negative,
                                                                                       ref.zero)
    assert factor.pivot_diagnostics.issue_count == ref.issue_count
    assert factor.pivot_diagnostics.equation_of_largest_ratio == ref.equation_of_largest
    assert factor.pivot_diagnostics.largest_ratio == pytest.approx(ref.largest_ratio, rel=1e-8)
    worst = 0.0
    for s in range(sym.supernode_count):
        mine, rows, _ = factor.panel(s)
        theirs, ref_rows, _ = ref.panel(s)
        assert np.array_equal(rows, ref_rows)
        scale = max(np.abs(theirs).max(), 1e-300)
        worst = max(worst, np.abs(mine - theirs).max() / scale)
    assert worst <= 1e-10, worst


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("columns", [1, 3, 64, 70])
def test_solve_matches_reference(name, columns, lib, oracle_mod, gpu):
    from o_o_solver_b200 import FactorSolve, SupernodalFactor

    model, sym, csc = build_case(name, oracle_mod)
    rng = np.random.default_rng(columns)
    b = np.asfortranarray(rng.standard_normal((sym.dof_count, columns)))
    if model.node_dofs == 6:
        b[:, : min(columns, 4)] = model.loads(sym.node_order, min(columns, 4))
    ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0)
    ref_avx = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=1)
    x_ref = ref.solve(b)
    spread = relative_columns(ref_avx.solve(b), x_ref).max()
    factor = SupernodalFactor.factorise(gpu_symbolic(sym), csc)
    x = np.asfortranarray(b.copy())
    FactorSolve(factor).solve(x)
    assert np.all(np.isfinite(x))
    assert residual(csc, x, b).max() <= 10.0 * residual(csc, x_ref, b).max() + 1e-13
    assert backward_error(csc, x, b).max() <= 1e-15
    difference = relative_columns(x, x_ref).max()
    print(f"{name}, {columns} columns: solution difference {difference:.2e} (reference families {spread:.2e})")
    assert difference <= solution_bound(spread), (difference, spread)


def test_device_entry_points(lib, oracle_mod, gpu):
    torch = gpu
    from o_o_solver_b200 import FactorSolve, SupernodalFactor, SymmetricCsc

    model, sym, csc = build_case("hex8", oracle_mod)
    dev = SymmetricCsc(torch.from_numpy(csc.offsets).cuda(), torch.from_numpy(csc.rows).cuda(),
                       torch.from_numpy(csc.values).cuda())
    factor = SupernodalFactor.factorise(gpu_symbolic(sym), dev)
    b = np.asfortranarray(np.random.default_rng(3).standard_normal((sym.dof_count, 5)))
    xb = torch.from_numpy(np.ascontiguousarray(b.T)).cuda().t()  # columns contiguous
    torch.cuda.synchronize()
    FactorSolve(factor).solve(xb)
    torch.cuda.synchronize()
    ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0)
    assert relative_columns(xb.cpu().numpy(), ref.solve(b)).max() < 1e-12


def test_refactorise_same_structure(lib, oracle_mod, gpu):
    from o_o_solver_b200 import FactorSolve, SupernodalFactor, SymmetricCsc

    model, sym, csc = build_case("hex8", oracle_mod)
    factor = SupernodalFactor.factorise(gpu_symbolic(sym), csc)
    scaled = SymmetricCsc(csc.offsets, csc.rows, csc.values * 3.0)
    factor.refactorise(scaled)
    b = np.asfortranarray(np.ones((sym.dof_count, 2)))
    x = b.copy(order="F")
    FactorSolve(factor).solve(x)
    ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, scaled.values, family=0)
    assert relative_columns(x, ref.solve(b)).max() < 1e-12


def test_zero_pivot_is_a_singularity(lib, oracle_mod, gpu):
    """A DOF without stiffness: SingularityError naming the first zero pivot, as the reference."""
    from o_o_solver_b200 import SingularityError, SupernodalFactor, SymmetricCsc

    model, sym, csc = build_case("plate6", oracle_mod)
    values = csc.values.copy()
    target = sym.dof_count // 3
    rows = csc.rows
    cols = np.repeat(np.arange(sym.dof_count), np.diff(csc.offsets))
    values[(rows == target) | (cols == target)] = 0.0
    bad = SymmetricCsc(csc.offsets, csc.rows, values)
    port = oracle_mod.PortFactor(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows, bad.offsets,
                                 bad.rows, bad.values)
    assert port.status > 0
    with pytest.raises(RuntimeError):
        oracle_mod.factorise(sym, bad.offsets, bad.rows, bad.values, family=0)
    factor = SupernodalFactor(gpu_symbolic(sym))
    with pytest.raises(SingularityError):
        factor.refactorise(bad)
    assert factor.zero_pivots[0] == port.zero_pivot_equation


def test_ratio_test_matches_reference(lib, oracle_mod, gpu):
    """MaxDiagonalRatio: the flagged pivots, their count and the largest ratio, with a bail-out < 0 (continue)."""
    from o_o_solver_b200 import FactorOptions, PivotPolicy, SupernodalFactor

    model, sym, csc = build_case("plate20", oracle_mod)
    ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0, max_ratio=1.0e2, bailout=-1)
    assert ref.issue_count > 0
    factor = SupernodalFactor.factorise(gpu_symbolic(sym), csc, FactorOptions(PivotPolicy(1.0e2, -1)))
    assert factor.pivot_diagnostics.issue_count == ref.issue_count
    assert factor.pivot_diagnostics.equation_of_largest_ratio == ref.equation_of_largest


def test_ratio_test_stops_with_bailout(lib, oracle_mod, gpu):
    from o_o_solver_b200 import FactorOptions, PivotPolicy, SingularityError, SupernodalFactor

    model, sym, csc = build_case("plate20", oracle_mod)
    with pytest.raises(RuntimeError):
        oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0, max_ratio=1.0e2, bailout=0)
    with pytest.raises(SingularityError):
        SupernodalFactor.factorise(gpu_symbolic(sym), csc, FactorOptions(PivotPolicy(1.0e2, 0)))


def test_negative_pivots_flagged(lib, oracle_mod, gpu):
    """An indefinite matrix in positive definite mode: the negative pivots are counted and flagged, as the
    reference does (MultifrontalDriver.cpp:810-817)."""
    from o_o_solver_b200 import FactorOptions, PivotPolicy, SupernodalFactor, SymmetricCsc

    model, sym, csc = build_case("hex4", oracle_mod)
    values = csc.values.copy()
    diagonal = csc.offsets[:-1]
    # An irrational share of the median diagonal: no pivot lands exactly on zero (a regular mesh repeats its
    # diagonal terms, and a shift of exactly half of them zeroes the corner DOFs' pivots).
    values[diagonal] -= 0.3781 * np.median(values[diagonal])
    shifted = SymmetricCsc(csc.offsets, csc.rows, values)
    ref = oracle_mod.factorise(sym, shifted.offsets, shifted.rows, shifted.values, family=0, bailout=-1)
    assert ref.negative > 0
    factor = SupernodalFactor.factorise(gpu_symbolic(sym), shifted, FactorOptions(PivotPolicy(1.0e7, -1)))
    assert (factor.inertia.positive, factor.inertia.negative) == (ref.positive, ref.negative)
    assert factor.pivot_diagnostics.issue_count == ref.issue_count


def test_entry_outside_structure_is_refused(lib, oracle_mod, gpu):
    from o_o_solver_b200 import SupernodalFactor, SymmetricCsc

    model, sym, csc = build_case("plate6", oracle_mod)
    rows = csc.rows.copy()
    # Column 0's last entry moved to a row the symbolic factor does not hold below column 0.
    last = csc.offsets[1] - 1
    held = set(sym.rows[sym.row_start[0]: sym.row_start[1]].tolist()) | set(range(sym.first_column[1]))
    outside = next(r for r in range(sym.dof_count - 1, 0, -1) if r not in held)
    rows[last] = outside
    with pytest.raises(ValueError):
        SupernodalFactor.factorise(gpu_symbolic(sym), SymmetricCsc(csc.offsets, rows, csc.values))


def test_solve_before_factorise_is_refused(lib, oracle_mod, gpu):
    from o_o_solver_b200 import FactorSolve, SupernodalFactor

    model, sym, csc = build_case("plate6", oracle_mod)
    factor = SupernodalFactor(gpu_symbolic(sym))
    with pytest.raises(RuntimeError):
        FactorSolve(factor).solve(np.zeros((sym.dof_count, 1), order="F"))


@pytest.mark.parametrize("name", ["plate100", "hex14"])
def test_refinement_reaches_tolerance(name, lib, oracle_mod, gpu):
    """FP64 refinement on the device stops on the normwise backward error: the device's own measure agrees with the
    host's, the refined solution's backward error is at the level of FP64 rounding, and its relative residual is no
    worse than the reference's solve's (the thin plate's floor is the cancellation in b - A x)."""
    from o_o_solver_b200 import SupernodalFactor, linalg

    model, sym, csc = build_case(name, oracle_mod)
    b = np.asfortranarray(np.random.default_rng(5).standard_normal((sym.dof_count, 9)))
    if model.node_dofs == 6:
        b[:, :4] = model.loads(sym.node_order, 4)
    factor = SupernodalFactor.factorise(gpu_symbolic(sym), csc)
    x = np.zeros_like(b, order="F")
    # A tolerance below what one solve reaches: the corrections run (at most 3).
    info = linalg.solve_refined(factor, b, x, tolerance=1.0e-18, max_steps=3)
    assert info.steps == 3
    host = backward_error(csc, x, b).max()
    assert host <= 1.0e-15, (host, info)
    assert info.backward_error == pytest.approx(host, rel=0.5)
    ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0)
    assert residual(csc, x, b).max() <= 2.0 * residual(csc, ref.solve(b), b).max() + 1e-14
    # The usual tolerance is met by the solve alone (no correction).
    info = linalg.solve_refined(factor, b, x, tolerance=1.0e-12)
    assert info.steps == 0 and info.backward_error <= 1.0e-12
    x_ref = ref.solve(b)
    # The refined solution is at least as close to the reference's as the reference's two kernel families are.
    spread = relative_columns(oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=1).solve(b),
                              x_ref).max()
    assert relative_columns(x, x_ref).max() <= solution_bound(spread)


def test_refinement_on_device_arrays(lib, oracle_mod, gpu):
    torch = gpu
    from o_o_solver_b200 import SupernodalFactor, linalg

    model, sym, csc = build_case("plate20", oracle_mod)
    factor = SupernodalFactor.factorise(gpu_symbolic(sym), csc)
    b = model.loads(sym.node_order, 3)
    d_b = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    d_x = torch.zeros_like(d_b)
    info = linalg.solve_refined(factor, d_b.t(), d_x.t(), tolerance=1.0e-12)
    torch.cuda.synchronize()
    assert backward_error(csc, d_x.cpu().numpy().T, b).max() <= 1.0e-15, info
    assert np.array_equal(d_b.cpu().numpy().T, b)  # B untouched


@pytest.mark.parametrize("name", ["hex14", "plate100"])
@pytest.mark.parametrize("mode", ["default", "alternative", "tune"])
def test_kernel_choices_match_reference(name, mode, lib, oracle_mod, gpu):
    """Both kernels of the launch kinds that have two (the diagonal blocks by sub-panels or by columns, the extend-add
    staged or element-wise), and the autotuner's mix of them, give the reference's factor: exact inertia, panels within
    1e-10; the autotuner reports a timed choice for each size class of those launches."""
    from o_o_solver_b200 import SupernodalFactor

    model, sym, csc = build_case(name, oracle_mod)
    ref = oracle_mod.factorise(sym, csc.offsets, csc.rows, csc.values, family=0)
    factor = SupernodalFactor(gpu_symbolic(sym))
    factor.set_tuning(mode)
    factor.refactorise(csc)
    factor.refactorise(csc)  # a replay of the recorded launches, with the choice made
    assert (factor.inertia.positive, factor.inertia.negative, factor.inertia.zero) == (ref.positive, ref.negative,
                                                                                       ref.zero)
    worst = 0.0
    for s in range(sym.supernode_count):
        mine, _, _ = factor.panel(s)
        theirs, _, _ = ref.panel(s)
        worst = max(worst, np.abs(mine - theirs).max() / max(np.abs(theirs).max(), 1e-300))
    assert worst <= 1e-10, worst
    report = factor.tuning()
    if mode == "tune":
        assert report and {r["kind"] for r in report} <= {"assemble_fronts", "diagonal_blocks", "update_matrix"}
        for r in report:
            assert r["launches"] > 0 and min(r["seconds"]) > 0.0 and r["chosen"] in (0, 1)
            assert r["seconds"][r["chosen"]] == min(r["seconds"])
    else:
        assert report == []
    factor.close()


def test_prefetched_right_hand_sides(lib, oracle_mod, gpu):
    """Loads prefetched before a refactorisation give the same solutions as loads uploaded by the solve; a prefetch of
    another array, or of the same array with other columns, is not used."""
    from o_o_solver_b200 import FactorSolve, SupernodalFactor

    model, sym, csc = build_case("plate20", oracle_mod)
    factor = SupernodalFactor(gpu_symbolic(sym))
    factor.refactorise(csc)
    b = np.asfortranarray(model.loads(sym.node_order, 5))
    plain = b.copy(order="F")
    FactorSolve(factor).solve(plain)
    ahead = b.copy(order="F")
    factor.prefetch(ahead)
    factor.refactorise(csc)
    FactorSolve(factor).solve(ahead)
    assert np.array_equal(ahead, plain)
    other = b.copy(order="F")
    factor.prefetch(np.asfortranarray(np.zeros_like(b)))
    FactorSolve(factor).solve(other)
    assert np.array_equal(other, plain)
    narrow = b[:, :3].copy(order="F")
    factor.prefetch(narrow)
    x = b[:, :3].copy(order="F")
    FactorSolve(factor).solve(x)
    assert np.array_equal(x, plain[:, :3])
    factor.close()
