"""Benchmark of the GPU hot path: the statics of the 580 x 580 shell plate (2,021,880 equations), factorisation of K
in the reference's symbolic order plus the solve of a 64-column load block, refined in FP64 until every column's
normwise backward error ||b - Ax||_inf / (||A||_inf ||x||_inf + ||b||_inf) is at most 1e-10 (the relative residual
||b - Ax||_2 / ||b||_2 is reported beside it: on this thin cantilever its FP64 floor is about 1e-5 for any solve, the
reference's included), on one B200 (replicas on N GPUs: every rank factorises and solves its own copy; no data-path
collective).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gpu|reference] [--workload plate580|plate100]

Prints one JSON line (rank 0). `value` is the device time of one step with its inputs resident in HBM (factorise +
solve + refinement), seconds; `e2e` the same step through the C ABI with host buffers (pinned), the copies included
(the loads prefetched on a copy stream while the matrix is factorised);
`roofline` the dominant kernel of a profiled factorisation against the measured peak; `cpu_baseline` the reference's
own factorisation and solve (oracle/_ref, built from its sources) on the host cores, on the same matrix.
`--impl reference` times that CPU path alone on the same workload.

The line's `modes` object is the other half of the metric: the lowest 20 modes of the 60^3 hexahedral block
(669,780 equations) by the GPU block shift-invert Lanczos (block 8), wall seconds of the whole solve (factorisations,
Lanczos runs, Sturm checks), its eigenvalues against the reference's recorded ones (tests/golden/modes), its e2e
through the public API from host arrays, and the reference beside it on the 30^3 block (a bounded CPU sample).

`forms.mixed` is the mixed-precision form on the same plate: the factorisation with its update matrices by 3xTF32
products on the tcgen05 tensor cores, the rate of that kernel beside the FP64 one, and FP64 GMRES refinement of its
solves (8 Krylov vectors, at most 3 corrections) with the backward error it reaches.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(ROOT, "tests", "golden", "orderings")

WORKLOADS = {
    # name: (plate size, right-hand sides)
    "plate580": (580, 64),
    "plate100": (100, 1),
    "plate200": (200, 64),
}


def parse():
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["gpu", "reference"], default="gpu")
    parser.add_argument("--workload", choices=sorted(WORKLOADS), default="plate580")
    parser.add_argument("--tolerance", type=float, default=1.0e-10)
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--modes-workload", choices=["hex60", "hex30", "hex14", "none"], default="hex60",
                        help="the modes leg: the lowest 20 modes of the n^3 hexahedral block, block size 8")
    parser.add_argument("--modes-steps", type=int, default=2)
    parser.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision form")
    parser.add_argument("--no-batched", action="store_true", help="skip the batched form")
    parser.add_argument("--batch-models", type=int, default=BATCH_MODELS)
    parser.add_argument("--batch-steps", type=int, default=3)
    parser.add_argument("--batch-reference-sample", type=int, default=16)
    parser.add_argument("--no-learned", action="store_true", help="skip the learned start block")
    parser.add_argument("--learned-train", type=int, default=192)
    parser.add_argument("--learned-test", type=int, default=64)
    parser.add_argument("--learned-epochs", type=int, default=3000)
    parser.add_argument("--factor-only", metavar="MODEL:PRECISION[:PIVOTING]", default=None,
                        help="factorise one model (plate<N> or hex<N> with an ordering under tests/golden/orderings; "
                             "precision fp64 or mixed) --steps times and print the factor's kernel statistics: the "
                             "small case for kernel captures")
    parser.add_argument("--launch-profile", metavar="PATH", default=None,
                        help="with --factor-only: also solve 64 load columns and write both launch lists (kind, "
                             "blocks, step column, device seconds) to PATH as JSON")
    parser.add_argument("--profile-rhs", type=int, default=64, help="with --launch-profile: the solve's columns")
    parser.add_argument("--kernels", choices=["tune", "default", "alternative"], default="tune",
                        help="the kernel choice of the launch kinds with two kernels (statics and --factor-only): the "
                             "autotuner's, or fixed; fixed for launch lists taken under ncu, whose serialised launches "
                             "would mislead the tuner's timing")
    parser.add_argument("--detail", metavar="PATH", default=None,
                        help="write the whole result record (kernel tables, every leg's detail) to PATH as JSON; "
                             "without it the record goes to stderr as one line")
    return parser.parse_args()


def load_workload(name):
    """The plate model, the reference's node order and supernode partition (tests/golden/orderings, made by the
    reference), the stiffness in that order and the load block."""
    from o_o_solver_b200 import workloads

    size, columns = WORKLOADS[name]
    fixture = np.load(os.path.join(GOLDEN, f"plate{size}.npz"))
    model = workloads.Model(workloads.PlateSpec(size, size))
    order = fixture["node_order"]
    csc = model.csc(order)
    loads = model.loads(order, columns)
    return model, fixture, csc, loads


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._thread = None

    def __enter__(self):
        def run():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.samples.append([v.strip() for v in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        sm_max = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 5 + k and "Active" in s[5 + k]
                          and "Not" not in s[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(sm_max) if sm_max else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp64_gemm_peak(torch, device):
    """The FP64 denominator: cuBLAS DGEMM (torch.matmul float64, 8192^3) throughput on this GPU, best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record()
        torch.matmul(a, b)
        stop.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (start.elapsed_time(stop) / 1e3))
    del a, b
    torch.cuda.empty_cache()
    return best / 1e12


def library_same_shapes(torch, device, symbolic, weights, fixture, small_order=128):
    """The update matrices of the factorisation done by the library instead: for every front above the small-front
    order with rows below its columns (c columns, r rows below), the product L_r L_r^T of an r x c block with itself,
    as one batched cuBLAS DGEMM (torch.bmm float64) per distinct (r, c), full r x r results (cuBLAS has no batched
    symmetric rank-k update). Device time of all the groups, best of 3, and its rate over the full products' 2 r^2 c
    flops; the fronts and their shapes come from the symbolic structure."""
    row_start, _ = symbolic.row_structure()
    r = np.diff(row_start)
    columns_before = np.concatenate([[0], np.cumsum(np.asarray(weights)[fixture["node_order"]])])
    first = np.asarray(fixture["first_position"])
    c = columns_before[first[1:]] - columns_before[first[:-1]]
    chosen = (c + r > small_order) & (r > 0)
    shapes = {}
    for rr, cc in zip(r[chosen].tolist(), c[chosen].tolist()):
        shapes[(rr, cc)] = shapes.get((rr, cc), 0) + 1
    groups = []
    for (rr, cc), count in shapes.items():
        per_batch = max(1, min(count, (1 << 27) // (rr * rr + rr * cc)))  # at most 1 GiB of operands and results
        for first_front in range(0, count, per_batch):
            batch = min(per_batch, count - first_front)
            groups.append(torch.randn(batch, rr, cc, dtype=torch.float64, device=device))
    flops = sum(2.0 * g.shape[0] * g.shape[1] * g.shape[1] * g.shape[2] for g in groups)
    best = None
    for _ in range(4):
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record()
        for g in groups:
            torch.bmm(g, g.transpose(1, 2))
        stop.record()
        torch.cuda.synchronize()
        seconds = start.elapsed_time(stop) / 1e3
        best = seconds if best is None else min(best, seconds)  # the first run warms cuBLAS up
    del groups
    torch.cuda.empty_cache()
    return {"fronts": int(chosen.sum()), "shapes": len(shapes), "ms": round(best * 1e3, 3),
            "tflops": round(flops / best / 1e12, 2)}


def accuracy(csc, x, b):
    """(largest relative residual ||b - Ax||_2/||b||_2, largest normwise backward error
    ||b - Ax||_inf / (||A||_inf ||x||_inf + ||b||_inf)) over the columns, on the host."""
    from o_o_solver_b200 import workloads

    r = b - workloads.lower_csc_multiply(csc, x)
    absolute = workloads.SymmetricCsc(csc.offsets, csc.rows, np.abs(csc.values))
    norm_a = workloads.lower_csc_multiply(absolute, np.ones((csc.dimension, 1)))[:, 0].max()
    residual = np.linalg.norm(r, axis=0) / np.linalg.norm(b, axis=0)
    backward = np.abs(r).max(axis=0) / (norm_a * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
    return float(residual.max()), float(backward.max())


def cpu_baseline(fixture, csc, loads, threads, graph):
    """The reference's factorisation + solve (oracle/_ref/liboos_ref.so) of the same matrix on the host cores. The
    matrix and loads may come from the package's generator or from oracle/plate_model.py (the same values bit for
    bit); the accuracy check is the oracle's own, so this leg loads nothing of the package."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import plate_model

    sym = oracle.analyse(*graph, given_order=fixture["node_order"], threads=threads)
    start = time.perf_counter()
    factor = oracle.factorise(sym, csc.offsets, csc.rows, csc.values, threads=threads)
    x = factor.solve(loads, threads=threads)
    seconds = time.perf_counter() - start
    resid, backward = plate_model.accuracy(plate_model.Csc(csc.offsets, csc.rows, csc.values), x, loads)
    return {"seconds": seconds, "factor_seconds": factor.seconds, "residual": resid, "backward_error": backward,
            "kernel": ["reference", "avx2", "avx512"][factor.kernel] if factor.kernel < 3 else str(factor.kernel)}


def load_modes_workload(name):
    """The hexahedral block, the reference's ordering and partition (tests/golden/orderings), K and the lumped M."""
    from o_o_solver_b200 import workloads

    size = int(name[3:])
    fixture = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    model = workloads.Model(workloads.HexSpec(size))
    order = fixture["node_order"]
    return model, fixture, model.csc(order, 0), model.csc(order, 1)


def reference_modes(name, threads):
    """The reference's SparsePencil + BlockLanczos::solve (oracle/_ref) of the same pencil: (seconds, eigenvalues)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    model, fixture, k, m = load_modes_workload(name)
    sym = oracle.analyse(model.offsets, model.neighbours, model.weights, given_order=fixture["node_order"],
                         threads=threads)
    result = oracle.modes(sym, k.offsets, k.rows, k.values, m.values, MODES, block_size=MODES_BLOCK, threads=threads,
                          vectors=False)
    return result["seconds"], result["eigenvalues"], result["factorisations"]


MODES = 20
MODES_BLOCK = 8


def gpu_modes(name, device, steps, warmup=1, e2e=False):
    """The lowest 20 modes on the GPU (SparsePencil + BlockLanczos, block 8): the median wall seconds of `steps`
    solves after `warmup`, the last solution, and with e2e the wall seconds of the public API from host arrays
    (the pencil built from the host CSC, the eigenvectors copied back)."""
    from o_o_solver_b200 import SparsePencil, SymbolicFactor
    from o_o_solver_b200.eigen import BlockLanczos, EigenRequest, LanczosOptions

    model, fixture, k, m = load_modes_workload(name)
    symbolic = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, fixture["node_order"],
                                             fixture["first_position"], fixture["parent"])
    pencil = SparsePencil(symbolic, k, m, device=device)
    solver = BlockLanczos(LanczosOptions(block_size=MODES_BLOCK))
    request = EigenRequest(mode_count=MODES)
    times = []
    solution = None
    for step in range(warmup + steps):
        solution = solver.solve(pencil, request, vectors=False)
        if step >= warmup:
            times.append(solution.seconds)
    result = {"seconds": statistics.median(times), "solution": solution, "symbolic": symbolic, "dimension": k.dimension}
    if e2e:
        import torch

        from o_o_solver_b200 import SymmetricCsc

        pencil.close()
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
        h_k = SymmetricCsc(pin(k.offsets), pin(k.rows), pin(k.values))
        h_m = SymmetricCsc(h_k.offsets, h_k.rows, pin(m.values))
        t0 = time.perf_counter()
        fresh = SparsePencil(symbolic, h_k, h_m, device=device)
        full = solver.solve(fresh, request, vectors=True)
        result["e2e"] = time.perf_counter() - t0
        result["h2d"] = int(k.offsets.nbytes + k.rows.nbytes + k.values.nbytes + m.values.nbytes)
        result["d2h"] = int(full.eigenvectors.nbytes + full.eigenvalues.nbytes)
        fresh.close()
    return result


def modes_leg(args, device, rank, world):
    """The modes half of the metric: GPU time of the lowest 20 modes of the workload, its accuracy against the
    reference's recorded eigenvalues (tests/golden/modes), the phases of the solve, and on one GPU the reference
    beside it on a bounded sample (the 30^3 block, seconds on the host cores)."""
    name = args.modes_workload
    run = gpu_modes(name, device, args.modes_steps, e2e=not args.no_e2e)
    solution = run["solution"]
    out = {"workload": f"{name}: {name[3:]}^3 trilinear hexahedra, base clamped, steel, lumped mass, "
                       f"{run['dimension']} equations; lowest {MODES} modes, block {MODES_BLOCK}",
           "value": run["seconds"], "unit": "s", "factorisations": solution.factorisation_count,
           "block_steps": solution.block_steps, "complete": solution.is_complete,
           "verified": solution.verified_count, "phases_s": {k: round(v, 4) for k, v in solution.phases.items()},
           "slow_paths": solution.slow_paths, "factor_device_s": round(solution.factor_seconds, 4)}
    golden = os.path.join(ROOT, "tests", "golden", "modes", f"{name}.npz")
    if os.path.exists(golden):
        expected = np.load(golden)["eigenvalues"]
        out["eigenvalue_max_rel_error_vs_reference"] = float(
            np.max(np.abs(solution.eigenvalues - expected) / np.abs(expected)))
        out["reference_recorded_s"] = float(np.load(golden)["seconds"])
        out["reference_recorded_threads"] = int(np.load(golden)["threads"])
    # Operator roofline: the solves read the factor twice (forward, backward) per block step.
    entries = run["symbolic"].factor_entry_count
    solves = solution.block_steps + sum(1 for r in solution.shifts if r.has_lanczos_run)
    if solution.phases.get("operator", 0.0) > 0.0 and solves > 0:
        bytes_per_solve = 2.0 * 8.0 * entries + 3.0 * 8.0 * run["dimension"] * MODES_BLOCK * 2
        out["operator_gbs"] = round(bytes_per_solve * solves / solution.phases["operator"] / 1e9, 1)
    if "e2e" in run:
        out["e2e"] = {"value": run["e2e"], "unit": "s", "h2d_bytes_per_step": run["h2d"],
                      "d2h_bytes_per_step": run["d2h"]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample = "hex30"
        try:
            threads = os.cpu_count() or 1
            ref_seconds, ref_values, ref_factorisations = reference_modes(sample, threads)
            gpu_sample = gpu_modes(sample, device, 1)
            out["cpu_baseline"] = {
                "value": ref_seconds, "unit": "s", "cores": threads, "kind": "reference",
                "sample": f"the same request on the 30^3 block (86,490 equations): reference "
                          f"{ref_seconds:.2f} s ({ref_factorisations} factorisations), GPU {gpu_sample['seconds']:.3f} s "
                          f"on that sample, eigenvalues agree to "
                          f"{float(np.max(np.abs(gpu_sample['solution'].eigenvalues - ref_values) / ref_values)):.1e}"}
        except Exception as error:  # the reference library is test infrastructure: absent, no baseline
            out["cpu_baseline"] = {"value": None, "unit": "s", "cores": 0, "kind": "reference",
                                   "sample": f"unavailable: {error}"}
    return out


def mixed_leg(factor, d_csc, d_loads, d_x, fp64_stats, tolerance, dev, torch):
    """The mixed-precision form on the same plate: the factorisation with its update matrices by 3xTF32 products on
    tcgen05 (device seconds, that kernel's rate beside the FP64 one), then FP64 refinement by GMRES corrections (8
    Krylov vectors, at most 3 corrections): the backward error it reaches and the time, against the FP64 solution."""
    from o_o_solver_b200 import FactorOptions, linalg

    options = FactorOptions(precision="mixed")
    factor.profile(True)
    factor.refactorise(d_csc, options)
    factor.refactorise(d_csc, options)
    stats = factor.kernel_stats()
    factor.profile(False)
    factor.refactorise(d_csc, options)
    factor_seconds = factor.device_seconds
    reference = d_x.clone()
    x = torch.empty_like(d_x)
    # One untimed refinement first: its Krylov workspace (9 vectors of the 64 columns, 9.3 GB) is allocated once.
    linalg.solve_refined(factor, d_loads.t(), x.t(), tolerance=tolerance, max_steps=3, krylov=8)
    torch.cuda.synchronize()
    start = time.perf_counter()
    info = linalg.solve_refined(factor, d_loads.t(), x.t(), tolerance=tolerance, max_steps=3, krylov=8)
    torch.cuda.synchronize()
    refine_seconds = time.perf_counter() - start
    difference = float(((x - reference).norm(dim=1) / reference.norm(dim=1)).max())
    um, um64 = stats["update_matrix"], fp64_stats["update_matrix"]
    factor.refactorise(d_csc)  # the FP64 factor back
    return {
        "factor_device_s": factor_seconds,
        "update_matrix": {"mixed_ms": round(um["seconds"] * 1e3, 3),
                          "mixed_tflops": round(um["flops"] / um["seconds"] / 1e12, 2),
                          "fp64_ms": round(um64["seconds"] * 1e3, 3),
                          "fp64_tflops": round(um64["flops"] / um64["seconds"] / 1e12, 2),
                          "kernel": "updateMatrixMixed: tcgen05.mma kind::tf32, 3 products, TMEM accumulator"},
        "gmres_ir": {"krylov": 8, "corrections": info.steps, "backward_error": info.backward_error,
                     "device_seconds": info.device_seconds,
                     "reaches_tolerance": bool(info.backward_error <= tolerance), "seconds": refine_seconds,
                     "max_rel_difference_vs_fp64_solution": difference},
        "step_s": factor_seconds + refine_seconds,
    }


# The kernel behind each kernel kind of the factorisation's statistics.
KERNEL_OF_KIND = {"small_fronts": "smallFronts", "assemble_fronts": "assembleFronts",
                  "diagonal_blocks": "diagonalBlocks", "panel_rows": "panelRowsInverse",
                  "panel_update": "panelUpdate", "update_matrix": "updateMatrix"}
TRAFFIC_TABLE = os.path.join(ROOT, "profiles", "dram_traffic.md")


def measured_traffic(kind, algorithmic_bytes_per_launch):
    """DRAM bytes per launch of a kernel kind: the ratio of ncu's dram__bytes_read.sum + dram__bytes_write.sum to the
    algorithmic bytes, measured on a capture small enough for the capture rules (profiles/dram_traffic.md, a row
    `| kernel | workload | dram bytes | algorithmic bytes | ratio |`), applied to this run's algorithmic bytes per
    launch. None when the kernel has no row."""
    kernel = KERNEL_OF_KIND.get(kind, kind)
    if not os.path.exists(TRAFFIC_TABLE):
        return None, None
    with open(TRAFFIC_TABLE) as table:
        for row in table:
            cells = [c.strip().strip("`") for c in row.strip().strip("|").split("|")]
            if len(cells) >= 5 and cells[0] == kernel:
                try:
                    ratio = float(cells[4])
                except ValueError:
                    continue
                return ratio * algorithmic_bytes_per_launch, f"{cells[1]}: {ratio:.3f} x the algorithmic bytes"
    return None, None


BATCH_MODELS = 512
BATCH_RHS = 8


def panel_fixture(cache={}):  # noqa: B006 (a cache of the reference's orderings by mesh size)
    def fixture_of(n):
        if n not in cache:
            cache[n] = dict(np.load(os.path.join(GOLDEN, f"panel{n}.npz")))
        return cache[n]

    return fixture_of


def batched_leg(args, dev, torch, replicas=None):
    """The batched form: BATCH_MODELS seeded stiffened panels (2,052 to 39,852 equations each, 4 to 12 blades,
    skin U[1, 4] mm), each with BATCH_RHS load cases, joined into one block-diagonal system (o_o_solver_b200.batch)
    and factorised and solved together, each factorisation and solve a replayed CUDA graph of launches: in FP64
    (`value`), and in the mixed form (update matrices by 3xTF32 products on tcgen05, then FP64 GMRES-IR to a backward
    error of 1e-10). Median device-timed seconds of the step over the steps; the backward error of every column of
    every panel checked on the host (the last form run, mixed); the reference on a sample of the panels (its time
    scaled by their share of the flops)."""
    from o_o_solver_b200 import FactorOptions, SupernodalFactor, SymmetricCsc, batch, linalg

    t0 = time.perf_counter()
    all_cases = batch.panel_cases(args.batch_models)
    # several GPUs: the panels dealt by their flops (longest first), each rank factorising its share
    rank, world = (replicas.rank, replicas.world) if replicas is not None else (0, 1)
    flops = [np.load(os.path.join(GOLDEN, f"panel{c.n}.npz"))["flops"] for c in all_cases]
    cases = [all_cases[i] for i in batch.deal(flops, world)[rank]]
    joined, rhs, parts = batch.panel_batch(cases, panel_fixture(), columns=BATCH_RHS)
    build_seconds = time.perf_counter() - t0
    d_csc = SymmetricCsc(torch.from_numpy(joined.matrix.offsets).to(dev), torch.from_numpy(joined.matrix.rows).to(dev),
                         torch.from_numpy(joined.matrix.values).to(dev))
    d_b = torch.from_numpy(np.ascontiguousarray(rhs.T)).to(dev)
    d_x = torch.empty_like(d_b)
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)

    def timed(options, krylov, max_steps, kernels="tune"):
        factor = SupernodalFactor(joined.symbolic, device=dev.index or 0)
        factor.set_tuning(kernels)
        factor.refactorise(d_csc, options)
        info = None
        for _ in range(max(args.warmup, 1)):  # the first runs also capture the graphs
            factor.refactorise(d_csc, options)
            info = linalg.solve_refined(factor, d_b.t(), d_x.t(), tolerance=1.0e-10, max_steps=max_steps,
                                        krylov=krylov)
        torch.cuda.synchronize()
        times = []
        for _ in range(args.batch_steps):
            start.record(torch.cuda.current_stream())
            factor.refactorise(d_csc, options)
            info = linalg.solve_refined(factor, d_b.t(), d_x.t(), tolerance=1.0e-10, max_steps=max_steps,
                                        krylov=krylov)
            stop.record(torch.cuda.current_stream())
            torch.cuda.synchronize()
            times.append(start.elapsed_time(stop) / 1e3)
        result = {"s": statistics.median(times), "factor_device_s": factor.device_seconds,
                  "refinement_steps": info.steps, "backward_error": info.backward_error,
                  "inertia_negative": factor.inertia.negative, "kernels": kernels, "tuning": factor.tuning()}
        factor.close()
        return result

    fixed = timed(FactorOptions(), 0, 10, kernels="default")
    fp64 = timed(FactorOptions(), 0, 10)
    mixed = timed(FactorOptions(precision="mixed"), 8, 3)
    if replicas is not None:
        fp64["s"] = replicas.slowest(fp64["s"])
        mixed["s"] = replicas.slowest(mixed["s"])
    seconds = fp64["s"]
    x = d_x.t().cpu().numpy()
    # every panel's normwise backward error per column, on the host
    worst = 0.0
    for part, xi, bi in zip(parts, joined.split(x), joined.split(rhs)):
        _, backward_error = accuracy(part.matrix, xi, bi)
        worst = max(worst, backward_error)
    out = {
        "workload": f"{len(cases)} seeded stiffened panels ({min(p.dof_count for p in parts)} to "
                    f"{max(p.dof_count for p in parts)} equations, 4-12 blades, skin U[1,4] mm), {BATCH_RHS} load "
                    "cases each, one block-diagonal factorisation",
        "models": len(all_cases), "ranks": world, "models_on_rank0": len(cases),
        "equations_on_rank0": joined.dimension, "flops_on_rank0": joined.symbolic.flop_count,
        "value": seconds, "unit": "s", "models_per_s": len(all_cases) / seconds,
        "form": "FP64 factorisation and solve (CUDA graphs), backward error checked at 1e-10",
        "fp64": fp64,
        "fp64_fixed_kernels": fixed,
        "mixed": dict(mixed, form="3xTF32 update matrices (tcgen05) + FP64 GMRES-IR (8 Krylov vectors, at most 3 "
                                  "corrections) to backward error 1e-10"),
        "max_backward_error_host": worst, "host_build_s": build_seconds,
    }
    # the reference on a sample of the panels, scaled by the flops (rank 0, on its share)
    sample = list(range(0, len(cases), max(1, len(cases) // args.batch_reference_sample)))
    if rank != 0:
        return out
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        from o_o_solver_b200 import workloads

        threads = os.cpu_count() or 1
        ref_seconds = 0.0
        sample_flops = 0.0
        fixture_of = panel_fixture()
        for i in sample:
            case = cases[i]
            fixture = fixture_of(case.n)
            model = workloads.Model(workloads.PanelSpec(n=case.n, stringers=case.stringers, thickness=case.thickness))
            sym = oracle.analyse(model.offsets, model.neighbours, model.weights, given_order=fixture["node_order"],
                                 threads=threads)
            part = parts[i]
            bi = np.asfortranarray(joined.split(rhs)[i])
            t1 = time.perf_counter()
            f = oracle.factorise(sym, part.matrix.offsets, part.matrix.rows, part.matrix.values, threads=threads)
            f.solve(bi, threads=threads)
            ref_seconds += time.perf_counter() - t1
            sample_flops += sym.flops
        out["cpu_baseline"] = {"value": ref_seconds * joined.symbolic.flop_count / sample_flops, "unit": "s",
                               "cores": threads, "kind": "reference",
                               "sample": f"{len(sample)} of the {len(cases)} panels factorised and solved one by one "
                                         f"({ref_seconds:.2f} s), scaled by their share of the flops"}
    except Exception as error:  # the reference library is test infrastructure: absent, no baseline
        out["cpu_baseline"] = {"value": None, "unit": "s", "cores": 0, "kind": "reference",
                               "sample": f"unavailable: {error}"}
    return out


LEARNED_MODES = 15


def wing_box(design):
    from o_o_solver_b200 import workloads

    return workloads.Model(workloads.WingBoxSpec(thicknesses=tuple(design)))


def learned_leg(args):
    """The learned start block on the wing box (span 10 m, chord 2 m, height 0.3 m, ribs every 0.5 m, shells of
    0.05 m: 133,800 equations), 24 zone thicknesses U[1, 4] mm: the lowest LEARNED_MODES modes of `learned_train`
    seeded designs by the solver with random starts, a network (24 -> 256 -> 256 -> 2,080) trained on the GPU on
    the projectors onto their modes' subspace in a 64-mode snapshot basis, then the `learned_test` unseen designs
    solved three ways: from the random start, from the learned start (the leading subspace of the predicted
    projector), and from the design's own modes perturbed by a seeded 1e-3 (relative) Gaussian, the start a perfect
    predictor with a small error would give (the ceiling of the method). Reported: the Lanczos seconds (the solve's
    wall time less its factorisations') and block steps of each, the agreement of the answers (eigenvalues, Sturm
    verification), how far the predicted subspace lies from the true one (sines of the principal angles in the
    design's own mass: the worst and the root mean square), and how much of the modes lies outside the snapshot
    basis at all (the least-squares residual in the design's mass, per mode)."""
    from o_o_solver_b200.learned import DesignSweep, LearnedStart, subspace_sines

    fixture = dict(np.load(os.path.join(GOLDEN, "wingbox.npz")))
    sweep = DesignSweep(wing_box, fixture, modes=LEARNED_MODES, block_size=8)
    rng = np.random.default_rng(0xB200)
    designs = rng.uniform(0.001, 0.004, (args.learned_train + args.learned_test, 24))
    train, test = designs[:args.learned_train], designs[args.learned_train:]
    t0 = time.perf_counter()
    solved = [sweep.solve(d) for d in train]
    data_seconds = time.perf_counter() - t0
    t1 = time.perf_counter()
    learned = LearnedStart.train(train, [s.eigenvectors for s, _ in solved], [m for _, m in solved], basis_size=64,
                                 block_size=8, hidden=256, epochs=args.learned_epochs, rate=1e-3)
    train_seconds = time.perf_counter() - t1
    noise = np.random.default_rng(0xA11CE)
    rows = []
    same = True

    def lanczos_seconds(solution):
        return solution.seconds - solution.phases["factorisation"]

    for d in test:
        plain, mass = sweep.solve(d, vectors=True)
        predicted = learned.predicted_modes(d)
        sines = subspace_sines(plain.eigenvectors, predicted, mass)
        outside = plain.eigenvectors - learned.basis.phi @ learned.basis.least_squares(plain.eigenvectors, mass)
        outside = np.sqrt(np.sum(mass[:, None] * outside * outside, axis=0))
        guided, _ = sweep.solve(d, start=learned.start_block(d), vectors=False)
        exact = plain.eigenvectors
        perturbed = exact + 1e-3 * noise.standard_normal(exact.shape) * np.sqrt(np.mean(exact * exact, axis=0))
        ceiling, _ = sweep.solve(d, start=np.ascontiguousarray((perturbed @ learned.mixing).T), vectors=False)
        for other in (guided, ceiling):
            same = same and plain.verified_count == other.verified_count and plain.is_complete == other.is_complete \
                and len(plain.eigenvalues) == len(other.eigenvalues)
        error = float(np.max(np.abs(guided.eigenvalues - plain.eigenvalues) / np.abs(plain.eigenvalues)))
        rows.append({"random_s": plain.seconds, "learned_s": guided.seconds,
                     "random_lanczos_s": lanczos_seconds(plain), "learned_lanczos_s": lanczos_seconds(guided),
                     "ceiling_lanczos_s": lanczos_seconds(ceiling),
                     "random_steps": plain.block_steps, "learned_steps": guided.block_steps,
                     "ceiling_steps": ceiling.block_steps,
                     "eigenvalue_rel_difference": error, "worst_sine": float(sines[-1]),
                     "rms_sine": float(np.sqrt(np.mean(sines ** 2))), "outside_basis_median": float(np.median(outside)),
                     "sturm": [(r.shift, r.sturm_count) for r in plain.shifts] == [(r.shift, r.sturm_count)
                                                                               for r in guided.shifts]})
    total = lambda key: sum(r[key] for r in rows)  # noqa: E731
    median = lambda key: float(np.median([r[key] for r in rows]))  # noqa: E731
    learned.network.close()
    return {
        "workload": f"wing box 10 m x 2 m x 0.3 m, ribs every 0.5 m, 0.05 m shells ({solved[0][1].shape[0]} "
                    f"equations), 24 zone thicknesses U[1,4] mm, lowest {LEARNED_MODES} modes, block 8",
        "train_designs": len(train), "test_designs": len(test), "basis": 64,
        "network": f"24 -> 256 -> 256 -> {64 * 65 // 2} (the projector onto the modes' subspace in the basis), "
                   f"FP32, Adam, {args.learned_epochs} epochs on the GPU",
        "final_loss": float(learned.losses[-1]), "initial_loss": float(learned.losses[0]),
        "data_s": data_seconds, "train_s": train_seconds,
        "lanczos_speedup": total("random_lanczos_s") / total("learned_lanczos_s"),
        "solve_speedup": total("random_s") / total("learned_s"),
        "block_steps": {"random": total("random_steps"), "learned": total("learned_steps"),
                        "ceiling": total("ceiling_steps")},
        "ceiling_lanczos_speedup": total("random_lanczos_s") / total("ceiling_lanczos_s"),
        # per design (robust to the occasional slow solve of either arm)
        "median_lanczos_speedup": float(np.median([r["random_lanczos_s"] / r["learned_lanczos_s"] for r in rows])),
        "median_ceiling_lanczos_speedup": float(np.median([r["random_lanczos_s"] / r["ceiling_lanczos_s"]
                                                           for r in rows])),
        "same_verification": bool(same), "same_sturm_points": all(r["sturm"] for r in rows),
        "max_eigenvalue_rel_difference": max(r["eigenvalue_rel_difference"] for r in rows),
        "median_worst_sine": median("worst_sine"), "median_rms_sine": median("rms_sine"),
        "median_outside_basis": median("outside_basis_median"),
        "per_design": rows,
    }


def run_reference(args, rank, world):
    """The reference's own CPU path on the workload: its factorisation and solve (oracle/_ref, built from the
    reference's sources) on all host cores. The plate, its node graph and its loads come from oracle/plate_model.py,
    so this process never loads the package's CUDA library. Under torchrun rank 0 alone runs; the others exit."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import plate_model

    size, columns = WORKLOADS[args.workload]
    fixture = dict(np.load(os.path.join(GOLDEN, f"plate{size}.npz")))
    plate = plate_model.Plate(size, size)
    csc = plate.csc(fixture["node_order"])
    loads = plate.loads(fixture["node_order"], columns)
    threads = os.cpu_count() or 1
    times = []
    result = None
    for step in range(args.warmup + args.steps):
        result = cpu_baseline(fixture, csc, loads, threads, (plate.offsets, plate.neighbours, plate.weights))
        if step >= args.warmup:
            times.append(result["seconds"])
    value = statistics.median(times)
    line = {
        "metric": metric_name(args.workload),
        "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded loads on a generated shell plate)",
        "config": {"workload": args.workload, "equations": int(csc.dimension), "rhs": int(loads.shape[1])},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "reference",
                         "sample": f"full {args.workload} factor + {loads.shape[1]}-column solve, kernel family "
                                   f"{result['kernel']}, residual {result['residual']:.2e}, backward error "
                                   f"{result['backward_error']:.1e}"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def metric_name(workload):
    if workload == "plate580":
        return "plate statics factor+solve time (2M-dof, 64 RHS)"
    return f"{workload} statics factor+solve time"


def run_gpu(args, rank, world, local_rank):
    import torch

    from o_o_solver_b200 import FactorSolve, SupernodalFactor, SymbolicFactor, SymmetricCsc, linalg, workloads

    torch.cuda.set_device(local_rank)
    from o_o_solver_b200.replicas import Replicas

    replicas = Replicas("nccl", timeout_s=600.0, device=torch.device("cuda", local_rank))

    model, fixture, csc, loads = load_workload(args.workload)
    n = csc.dimension
    columns = loads.shape[1]
    symbolic = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, fixture["node_order"],
                                             fixture["first_position"], fixture["parent"])
    factor = SupernodalFactor(symbolic, device=local_rank)
    factor.set_tuning(args.kernels)
    stream = torch.cuda.ExternalStream(factor.stream)
    dev = torch.device("cuda", local_rank)
    d_csc = SymmetricCsc(torch.from_numpy(csc.offsets).to(dev), torch.from_numpy(csc.rows).to(dev),
                         torch.from_numpy(csc.values).to(dev))
    d_loads = torch.from_numpy(np.ascontiguousarray(loads.T)).to(dev)  # (columns, n): columns contiguous
    d_x = torch.empty_like(d_loads)
    torch.cuda.synchronize()
    solver = FactorSolve(factor)

    refinement = {}

    def step():
        factor.refactorise(d_csc)
        info = linalg.solve_refined(factor, d_loads.t(), d_x.t(), tolerance=args.tolerance, max_steps=10)
        refinement["steps"] = info.steps
        refinement["residual"] = info.residual
        refinement["backward_error"] = info.backward_error
        refinement["solve_seconds"] = info.device_seconds
        refinement["factor_seconds"] = factor.device_seconds

    for _ in range(args.warmup):
        step()  # the first also runs the autotuner's timing factorisations
    torch.cuda.synchronize()
    tuning = factor.tuning()
    replicas.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        stop.record(stream)
        torch.cuda.synchronize()
    replicas.barrier()
    torch.cuda.synchronize()
    seconds = replicas.slowest(start.elapsed_time(stop) / 1e3 / args.steps)

    # Residual of the last step's solutions (host check of the device's own test).
    x = d_x.t().cpu().numpy()
    resid, backward = accuracy(csc, x, loads)
    factor_launches, solve_launches = factor.launch_counts(columns)
    launches = args.steps * (factor_launches + solve_launches * (1 + refinement.get("steps", 0)))

    # End to end through the C ABI with host (pinned) buffers.
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
        h_offsets, h_rows, h_values = pin(csc.offsets), pin(csc.rows), pin(csc.values)
        h_csc = SymmetricCsc(h_offsets, h_rows, h_values)
        h_b = torch.from_numpy(np.ascontiguousarray(loads.T)).pin_memory().numpy().T  # pinned, column-major
        h_x = torch.empty((columns, n), dtype=torch.float64).pin_memory().numpy().T
        e2e_times = []
        for k in range(max(1, min(3, args.steps)) + 1):
            t0 = time.perf_counter()
            factor.prefetch(h_b)  # the loads travel while the matrix is factorised
            factor.refactorise(h_csc)
            linalg.solve_refined(factor, h_b, h_x, tolerance=args.tolerance, max_steps=10)
            if k > 0:
                e2e_times.append(time.perf_counter() - t0)
        h2d = csc.offsets.nbytes + csc.rows.nbytes + csc.values.nbytes + loads.nbytes
        e2e = {"value": statistics.median(e2e_times), "unit": "s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(loads.nbytes)}

    # Roofline of the dominant kernel: one profiled factorisation.
    factor.profile(True)
    factor.refactorise(d_csc)
    stats = factor.kernel_stats()
    factor.profile(False)
    dominant = max(stats, key=lambda k: stats[k]["seconds"])
    d = stats[dominant]
    peaks, peak_source = measured_peaks()
    compute_bound = dominant in ("panel_update", "update_matrix", "panel_rows", "diagonal_blocks")
    if compute_bound:
        fp64 = fp64_gemm_peak(torch, dev)
        achieved = d["flops"] / d["seconds"] / 1e12
        traffic, traffic_source = measured_traffic(dominant, d["bytes"] / d["launches"])
        roofline = {"bound": "tensor", "achieved": achieved, "peak": fp64, "unit": "TFLOP/s", "frac": achieved / fp64,
                    "traffic": traffic, "traffic_source": traffic_source,
                    "algorithmic_bytes_per_launch": d["bytes"] / d["launches"],
                    "kernel": dominant, "launches": d["launches"],
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor)",
                    "share": d["seconds"] / sum(v["seconds"] for v in stats.values())}
        if dominant == "update_matrix":
            # The same update matrices by the library, against this kernel's own event time (`ms`).
            roofline["library_same_shapes"] = {
                **library_same_shapes(torch, dev, symbolic, model.weights, fixture),
                "kernel_ms": round(d["seconds"] * 1e3, 3)}
    else:
        achieved = d["bytes"] / d["seconds"] / 1e9
        traffic, traffic_source = measured_traffic(dominant, d["bytes"] / d["launches"])
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "traffic_source": traffic_source,
                    "kernel": dominant,
                    "launches": d["launches"], "peak_source": f"hbm_gbs ({peak_source})",
                    "share": d["seconds"] / sum(v["seconds"] for v in stats.values())}
    kernel_table = {k: {"ms": round(v["seconds"] * 1e3, 3), "launches": v["launches"],
                        "tflops": round(v["flops"] / v["seconds"] / 1e12, 3) if v["seconds"] > 0 else None,
                        "gbs": round(v["bytes"] / v["seconds"] / 1e9, 1) if v["seconds"] > 0 else None}
                    for k, v in stats.items()}

    baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            cb = cpu_baseline(fixture, csc, loads, threads, (model.offsets, model.neighbours, model.weights))
            baseline = {"value": cb["seconds"], "unit": "s", "cores": threads, "kind": "reference",
                        "sample": f"one full {args.workload} factor + {columns}-column solve "
                                  f"({cb['kernel']} kernels, factor {cb['factor_seconds']:.3f} s, "
                                  f"residual {cb['residual']:.2e}, backward error {cb['backward_error']:.1e})"}
        except Exception as error:  # the reference library is test infrastructure: absent, no baseline
            baseline = {"value": None, "unit": "s", "cores": 0, "kind": "reference", "sample": f"unavailable: {error}"}

    modes = modes_leg(args, local_rank, rank, world) if args.modes_workload != "none" else None
    mixed = None if args.no_mixed else mixed_leg(factor, d_csc, d_loads, d_x, stats, args.tolerance, dev, torch)
    batched = None if args.no_batched else batched_leg(args, dev, torch, replicas)
    learned = None if args.no_learned else learned_leg(args)

    if rank == 0:
        line = {
            "metric": metric_name(args.workload),
            "value": seconds, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": seconds * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded loads on a generated shell plate)",
            "config": {"workload": args.workload, "equations": n, "rhs": columns, "form": "plain FP64",
                       "flops_per_factor": symbolic.flop_count, "l2": "inputs larger than L2 (panels 6 GB)",
                       "parallelism": f"replicas x{world}" if world > 1 else "one GPU"},
            "residual": resid, "backward_error": backward, "refinement": refinement, "e2e": e2e,
            "gpu_launches": launches, "roofline": roofline, "kernels": kernel_table, "clocks": clocks.summary(),
            "cpu_baseline": baseline, "factor_tflops": symbolic.flop_count / refinement["factor_seconds"] / 1e12,
            "tuning": tuning,
            "modes": modes, "forms": {"mixed": mixed, "batched": batched, "learned_start": learned},
        }
        emit(line, args.detail)
    replicas.close()


def _round(value, digits=4):
    if isinstance(value, float):
        return float(f"{value:.{digits}g}")
    if isinstance(value, dict):
        return {k: _round(v, digits) for k, v in value.items()}
    if isinstance(value, list):
        return [_round(v, digits) for v in value]
    return value


def _pick(source, *keys):
    if not source:
        return None
    return {k: source[k] for k in keys if k in source}


def compact_line(full):
    """The final stdout line: the fields a reader of the result needs, a few numbers per leg, well under 4 KB.
    Everything else (kernel tables, per-design rows, phases) goes to the detail record."""
    line = {k: full[k] for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                                 "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config")}
    line.update({k: full.get(k) for k in ("residual", "backward_error", "e2e", "gpu_launches", "clocks",
                                          "cpu_baseline", "factor_tflops")})
    line["refinement"] = _pick(full.get("refinement"), "steps", "factor_seconds", "solve_seconds")
    line["roofline"] = _pick(full.get("roofline"), "bound", "achieved", "peak", "unit", "frac", "traffic", "kernel",
                             "launches", "share", "peak_source", "library_same_shapes")
    modes = full.get("modes")
    if modes:
        line["modes"] = _pick(modes, "value", "unit", "factorisations", "block_steps", "verified",
                              "eigenvalue_max_rel_error_vs_reference", "operator_gbs")
        if modes.get("e2e"):
            line["modes"]["e2e"] = modes["e2e"]["value"]
        if modes.get("cpu_baseline"):
            line["modes"]["cpu_baseline"] = _pick(modes["cpu_baseline"], "value", "cores", "kind", "sample")
    forms = full.get("forms") or {}
    compact_forms = {}
    if forms.get("mixed"):
        m = forms["mixed"]
        compact_forms["mixed"] = {"step_s": m.get("step_s"), "factor_device_s": m.get("factor_device_s"),
                                  **_pick(m.get("gmres_ir"), "device_seconds", "backward_error", "reaches_tolerance",
                                          "corrections", "max_rel_difference_vs_fp64_solution")}
    if forms.get("batched"):
        b = forms["batched"]
        compact_forms["batched"] = {**_pick(b, "value", "models_per_s", "models", "max_backward_error_host"),
                                    "fixed_kernels_s": (b.get("fp64_fixed_kernels") or {}).get("s"),
                                    "mixed_s": (b.get("mixed") or {}).get("s"),
                                    "cpu_baseline": (b.get("cpu_baseline") or {}).get("value")}
    if forms.get("learned_start"):
        compact_forms["learned_start"] = _pick(forms["learned_start"], "lanczos_speedup", "median_lanczos_speedup",
                                               "ceiling_lanczos_speedup", "same_verification", "same_sturm_points",
                                               "max_eigenvalue_rel_difference")
    line["forms"] = compact_forms
    return _round(line)


def emit(full, detail_path):
    """Write the whole record (to `detail_path`, else as one line on stderr) and print the compact line last."""
    if detail_path:
        with open(detail_path, "w") as out:
            json.dump(full, out, indent=1)
    else:
        print(json.dumps(full), file=sys.stderr, flush=True)
    print(json.dumps(compact_line(full)), flush=True)


def factor_only(args):
    """Factorise one model --steps times (after --warmup untimed ones) on cuda:0 and print its kernel statistics."""
    import torch

    from o_o_solver_b200 import FactorOptions, SupernodalFactor, SymbolicFactor, workloads

    name, _, rest = args.factor_only.partition(":")
    precision, _, pivoting = rest.partition(":")
    kind = "plate" if name.startswith("plate") else "hex"
    size = int(name[len(kind):])
    fixture = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    model = workloads.Model(workloads.PlateSpec(size, size) if kind == "plate" else workloads.HexSpec(size))
    order = fixture["node_order"]
    symbolic = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, order,
                                             fixture["first_position"], fixture["parent"])
    options = FactorOptions(precision=precision or "fp64", pivoting=pivoting or "positive_definite")
    stiffness = model.csc(order, 0)
    torch.cuda.init()
    factor = SupernodalFactor(symbolic)
    factor.set_tuning(args.kernels)
    factor.refactorise(stiffness, options)
    for _ in range(max(args.warmup - 1, 0)):
        factor.refactorise(stiffness, options)
    factor.profile(True)
    start = time.perf_counter()
    for _ in range(args.steps):
        factor.refactorise(stiffness, options)
    seconds = (time.perf_counter() - start) / max(args.steps, 1)
    if args.launch_profile:
        from o_o_solver_b200 import linalg

        loads = torch.from_numpy(np.ascontiguousarray(model.loads(order, args.profile_rhs).T)).to("cuda")
        x = torch.empty_like(loads)
        linalg.solve_refined(factor, loads.t(), x.t(), tolerance=1.0, max_steps=0)
        torch.cuda.synchronize()
        with open(args.launch_profile, "w") as out:
            json.dump({"factor": factor.launch_profile("factor"), "solve": factor.launch_profile("solve")}, out)
    print(json.dumps({"factor_only": name, "precision": options.precision, "equations": int(symbolic.dof_count),
                      "kernel_choice": args.kernels, "wall_seconds_per_factor": seconds,
                      "kernels": factor.kernel_stats(), "tuning": factor.tuning()}), flush=True)
    factor.close()


def main():
    args = parse()
    if args.factor_only:
        factor_only(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
