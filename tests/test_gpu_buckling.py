"""The buckling solve on the GPU (BlockLanczos::solveBuckling over a BucklingPencil) against the reference's own solve
of the same pencil: K phi = lambda B phi with B = -K_d, K a plate's or a solid's stiffness and K_d a differential
stiffness of membrane loads on its pattern (compression along one axis and tension along another on the plate, so
that load factors of both signs answer). The load factors nearest 0 within 1e-9 relative (or three times the spread
between two of the reference's kernel families), the same shifts with the same purposes and Sturm counts as the
reference's walk, every count the reference's inertia of that shift, the eigenvectors K-orthonormal with small
residuals, and the reference's refusals."""

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

EIGENVALUE_TOLERANCE = 1e-9
# (kind, size, membrane line loads N_x, N_y, N_z, displacement components they act on)
LOADS = {"plate": ((-1000.0, 300.0, 0.0), (2,)), "hex": ((0.0, 0.0, -1.0e9), (0, 1, 2))}


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def problem(kind, size, oracle):
    from o_o_solver_b200 import SymbolicFactor, workloads

    model = workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))
    sym = oracle.analyse(model.offsets, model.neighbours, model.weights, model.coordinates)
    k = model.csc(sym.node_order, 0)
    loads, components = LOADS[kind]
    kd = model.differential(sym.node_order, k, line_loads=loads, components=components)
    symbolic = SymbolicFactor.from_arrays(sym.dof_count, sym.first_column, sym.parent, sym.row_start, sym.rows)
    return sym, symbolic, k, kd


def sturm_count(oracle, sym, k, kd, sigma):
    """The reference's negative pivots of S (K + sigma K_d) S (S the pencil scale of K)."""
    scale = oracle.pencil_scale(k.offsets, k.rows, k.values)
    cols = np.repeat(np.arange(k.dimension), np.diff(k.offsets))
    values = (k.values + sigma * kd.values) * scale[k.rows] * scale[cols]
    return oracle.factorise(sym, k.offsets, k.rows, values, indefinite=True, family=0).negative


def pair_figures(k, kd, values, vectors):
    """Per pair: ||K phi + lambda K_d phi|| / ||K phi||, and how far lambda lies from the Rayleigh quotient of its
    vector, relatively; and phi^T K phi."""
    from o_o_solver_b200 import workloads

    kphi = workloads.lower_csc_multiply(k, vectors)
    kdphi = workloads.lower_csc_multiply(kd, vectors)
    residual = np.linalg.norm(kphi + kdphi * values, axis=0) / np.linalg.norm(kphi, axis=0)
    quotient = np.einsum("ij,ij->j", vectors, kphi) / -np.einsum("ij,ij->j", vectors, kdphi)
    return residual, np.abs(quotient - values) / np.abs(values), vectors.T @ kphi


def check_pairs(k, kd, values, vectors, reference):
    """K-orthonormal eigenvectors whose residuals are at most 1e-8, or ten times the reference's largest residual of
    the same request (a thin plate's K amplifies the vectors' rounding in ||K phi + lambda K_d phi|| and in
    phi^T K phi: the reference's own pairs of the 40 x 40 plate reach 3.4e-6)."""
    residual, _, gram = pair_figures(k, kd, values, vectors)
    theirs, _, their_gram = pair_figures(k, kd, *reference)
    bound = max(1e-8, 10.0 * theirs.max())
    assert np.all(residual <= bound), (residual, bound)
    # the K-inner products cancel the same way: the reference's vectors are K-orthonormal to 7e-9 on the 40 x 40 plate
    assert np.abs(gram - np.eye(len(values))).max() <= max(1e-10, 10.0 * np.abs(their_gram - np.eye(len(values))).max())


def reference(oracle, sym, k, kd, count, block, lower=-np.inf, upper=np.inf, family=-1, vectors=False):
    return oracle.modes(sym, k.offsets, k.rows, k.values, kd.values, count, block_size=block, family=family,
                        vectors=vectors, lower=lower, upper=upper, buckling=True, capacity=max(count, 64))


def compare(solution, ref, oracle, sym, k, kd, spread):
    """The load factors within 1e-9 relative, or three times the spread of the reference's kernel families, or ten
    times how far either solve's value lies from its vector's Rayleigh quotient (the K-inner products of a thin
    plate's softest modes cancel: the reference's 11th root of the 40 x 40 plate is 3.2e-8 from its own quotient,
    with both families agreeing to 2e-8 because they share the sparse products)."""
    assert solution.is_complete == ref["complete"]
    assert len(solution.eigenvalues) == len(ref["eigenvalues"])
    relative = np.abs(solution.eigenvalues - ref["eigenvalues"]) / np.abs(ref["eigenvalues"])
    _, mine, _ = pair_figures(k, kd, solution.eigenvalues, solution.eigenvectors)
    _, theirs, _ = pair_figures(k, kd, ref["eigenvalues"], ref["eigenvectors"])
    bound = np.maximum(max(EIGENVALUE_TOLERANCE, 3.0 * spread), 10.0 * np.maximum(mine, theirs))
    print(f"largest relative difference {relative.max():.2e} (reference families {spread:.2e}, quotients "
          f"{mine.max():.2e} / {theirs.max():.2e})")
    assert np.all(relative <= bound), (relative, bound)
    # the same walk: shifts, purposes and Sturm counts
    assert solution.factorisation_count == ref["factorisations"]
    assert len(solution.shifts) == len(ref["shifts"])
    purposes = ["lowest_bound", "lower_bound", "upper_bound", "advance", "fill_gap"]
    for record, row in zip(solution.shifts, ref["shifts"]):
        assert record.purpose == purposes[int(row[1])], (record, row)
        assert record.sturm_count == int(row[2]), (record, row)
        assert record.has_lanczos_run == bool(row[3]), (record, row)
        assert abs(record.shift - row[0]) <= 1e-6 * max(abs(row[0]), 1e-300), (record, row)
        assert record.sturm_count == sturm_count(oracle, sym, k, kd, record.shift), record


@pytest.mark.parametrize("kind,size,count,block", [("plate", 20, 10, 8), ("plate", 40, 12, 7), ("hex", 8, 10, 8)])
def test_load_factors_match_reference(kind, size, count, block, lib, oracle_mod, gpu):
    from o_o_solver_b200 import BucklingPencil
    from o_o_solver_b200.eigen import BlockLanczos, EigenRequest, LanczosOptions

    sym, symbolic, k, kd = problem(kind, size, oracle_mod)
    ref = reference(oracle_mod, sym, k, kd, count, block, vectors=True)
    families = [reference(oracle_mod, sym, k, kd, count, block, family=f)["eigenvalues"] for f in (0, 1)]
    spread = (np.abs(families[0] - families[1]) / np.abs(families[1])).max()
    pencil = BucklingPencil(symbolic, k, kd)
    solution = BlockLanczos(LanczosOptions(block_size=block)).solve(pencil, EigenRequest(mode_count=count))
    assert solution.is_complete and solution.verified_count == count
    magnitudes = np.abs(solution.eigenvalues)
    assert np.all(np.diff(magnitudes) >= 0)
    if kind == "plate":
        assert (solution.eigenvalues > 0).any() and (solution.eigenvalues < 0).any()
    compare(solution, ref, oracle_mod, sym, k, kd, spread)
    assert np.all(solution.residual_bounds <= 1e-10)
    check_pairs(k, kd, solution.eigenvalues, solution.eigenvectors, (ref["eigenvalues"], ref["eigenvectors"]))
    assert solution.factorisation_count == pencil.factorisation_count
    pencil.close()


def test_range_request(lib, oracle_mod, gpu):
    """Both bounds and no count: every load factor in [-0.16, 0.2), the counts at the bounds factorised first."""
    from o_o_solver_b200 import BucklingPencil
    from o_o_solver_b200.eigen import BlockLanczos, EigenRequest, LanczosOptions

    sym, symbolic, k, kd = problem("plate", 20, oracle_mod)
    ref = reference(oracle_mod, sym, k, kd, 0, 8, lower=-0.16, upper=0.2, vectors=True)
    families = [reference(oracle_mod, sym, k, kd, 0, 8, lower=-0.16, upper=0.2, family=f)["eigenvalues"]
                for f in (0, 1)]
    spread = (np.abs(families[0] - families[1]) / np.abs(families[1])).max()
    pencil = BucklingPencil(symbolic, k, kd)
    solution = BlockLanczos(LanczosOptions(block_size=8)).solve(
        pencil, EigenRequest(lower_bound=-0.16, upper_bound=0.2, mode_count=0))
    assert len(solution.eigenvalues) > 0
    assert np.all((solution.eigenvalues >= -0.16) & (solution.eigenvalues < 0.2))
    compare(solution, ref, oracle_mod, sym, k, kd, spread)
    pencil.close()


def test_refusals(lib, oracle_mod, gpu):
    """An indefinite K (K + 0.1 K_d, past the lowest load factor: SolverError at the factorisation at 0, as the
    reference) and a request with neither a count nor both bounds (ValueError)."""
    from o_o_solver_b200 import BucklingPencil, SolverError, SymmetricCsc
    from o_o_solver_b200.eigen import BlockLanczos, EigenRequest

    sym, symbolic, k, kd = problem("plate", 12, oracle_mod)
    unstable = SymmetricCsc(k.offsets, k.rows, k.values + 0.1 * kd.values)
    with pytest.raises(RuntimeError, match="not positive definite"):  # the reference refuses it too
        reference(oracle_mod, sym, unstable, kd, 4, 8)
    pencil = BucklingPencil(symbolic, unstable, kd)
    with pytest.raises(SolverError):
        BlockLanczos().solve(pencil, EigenRequest(mode_count=4))
    pencil.close()
    pencil = BucklingPencil(symbolic, k, kd)
    with pytest.raises(ValueError):
        BlockLanczos().solve(pencil, EigenRequest(mode_count=0))
    pencil.close()
