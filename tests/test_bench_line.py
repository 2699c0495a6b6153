"""The benchmark's output contract on the CPU: the final line stays small and parseable whatever the legs report,
and the reference arm runs the reference's own CPU path without loading anything of the package."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

REQUIRED = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "roofline", "cpu_baseline", "clocks")


def full_record():
    """A record as large as the GPU arm writes: every leg, the kernel table, 64 per-design rows."""
    row = {"random_s": 0.2789235, "learned_s": 0.2320576, "random_lanczos_s": 0.2299735, "learned_lanczos_s": 0.184067,
           "ceiling_lanczos_s": 0.1221534, "random_steps": 28, "learned_steps": 28, "ceiling_steps": 18,
           "eigenvalue_rel_difference": 9.0e-15, "worst_sine": 0.99999994, "rms_sine": 0.8635, "sturm": False}
    kernels = {k: {"ms": 12.345678, "launches": 253, "tflops": 11.812345, "gbs": 666.123} for k in bench.KERNEL_OF_KIND}
    return {
        "metric": bench.metric_name("plate580"), "value": 0.1153, "unit": "s", "n_gpus": 1, "steps": 20, "warmup": 5,
        "ms_per_step": 115.3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded loads on a generated shell plate)",
        "config": {"workload": "plate580", "equations": 2021880, "rhs": 64, "form": "plain FP64",
                   "flops_per_factor": 8.32e11, "l2": "inputs larger than L2 (panels 6 GB)", "parallelism": "one GPU"},
        "residual": 1.88e-05, "backward_error": 1.8e-16,
        "refinement": {"steps": 0, "residual": 1.9e-5, "backward_error": 1.8e-16, "solve_seconds": 0.0322,
                       "factor_seconds": 0.0825},
        "e2e": {"value": 0.167, "unit": "s", "h2d_bytes_per_step": 700000000, "d2h_bytes_per_step": 1035202560},
        "gpu_launches": 21000,
        "roofline": {"bound": "tensor", "achieved": 21.6, "peak": 35.5, "unit": "TFLOP/s", "frac": 0.61,
                     "traffic": 1.19e9, "traffic_source": "hex30: 1.280 x the algorithmic bytes",
                     "algorithmic_bytes_per_launch": 9.3e8, "kernel": "update_matrix", "launches": 16,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor)", "share": 0.3,
                     "library_same_shapes": {"fronts": 17091, "shapes": 182, "ms": 39.442, "tflops": 29.63,
                                             "kernel_ms": 25.365}},
        "kernels": kernels,
        "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 40},
        "cpu_baseline": {"value": 4.957, "unit": "s", "cores": 16, "kind": "reference",
                         "sample": "one full plate580 factor + 64-column solve (avx2 kernels, factor 4.1 s, residual "
                                   "1.88e-05, backward error 2.2e-15)"},
        "factor_tflops": 10.1,
        "modes": {"workload": "hex60: 60^3 trilinear hexahedra " * 3, "value": 1.96, "unit": "s", "factorisations": 4,
                  "block_steps": 31, "complete": True, "verified": 20,
                  "phases_s": {"factorisation": 0.95, "operator": 0.73, "orthogonalisation": 0.08},
                  "factor_device_s": 0.9, "eigenvalue_max_rel_error_vs_reference": 1.2e-12,
                  "reference_recorded_s": 270.0, "operator_gbs": 651.0,
                  "e2e": {"value": 2.35, "unit": "s", "h2d_bytes_per_step": 1, "d2h_bytes_per_step": 2},
                  "cpu_baseline": {"value": 3.13, "unit": "s", "cores": 16, "kind": "reference",
                                   "sample": "the same request on the 30^3 block (86,490 equations): reference 3.13 s "
                                             "(4 factorisations), GPU 0.261 s on that sample, eigenvalues agree to "
                                             "1.0e-12"}},
        "forms": {
            "mixed": {"factor_device_s": 0.0813, "update_matrix": {"mixed_ms": 22.3}, "step_s": 1.25,
                      "gmres_ir": {"krylov": 8, "corrections": 3, "backward_error": 8.9e-10, "reaches_tolerance": False,
                                   "seconds": 1.2, "max_rel_difference_vs_fp64_solution": 1.06}},
            "batched": {"workload": "512 seeded stiffened panels " * 4, "models": 512, "value": 0.174,
                        "models_per_s": 2943.0, "fp64": {"s": 0.174}, "mixed": {"s": 0.95},
                        "max_backward_error_host": 6.6e-10,
                        "cpu_baseline": {"value": 11.5, "unit": "s", "cores": 16, "kind": "reference", "sample": "x" * 200}},
            "learned_start": {"lanczos_speedup": 1.07, "median_lanczos_speedup": 1.03, "ceiling_lanczos_speedup": 1.5,
                              "same_verification": True, "same_sturm_points": False,
                              "max_eigenvalue_rel_difference": 5.3e-14, "per_design": [row] * 64},
        },
    }


def test_compact_line_is_small_and_complete():
    line = json.dumps(bench.compact_line(full_record()))
    assert len(line) < 4096, len(line)
    parsed = json.loads(line)
    for key in REQUIRED:
        assert key in parsed, key
    assert parsed["value"] > 0 and parsed["config"]["workload"] == "plate580"
    assert "per_design" not in line and "kernels" not in parsed


def test_emit_prints_the_compact_line_last(tmp_path, capsys):
    detail = tmp_path / "detail.json"
    bench.emit(full_record(), str(detail))
    out = capsys.readouterr().out.strip().splitlines()
    assert json.loads(out[-1])["metric"] == bench.metric_name("plate580")
    assert len(json.loads(detail.read_text())["forms"]["learned_start"]["per_design"]) == 64


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "liboos_ref.so")),
                    reason="the reference oracle is not built")
def test_reference_arm_loads_nothing_of_the_package():
    script = (
        "import runpy, sys, json\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'plate100', '--steps', '1', '--warmup', '0']\n"
        f"runpy.run_path({os.path.join(ROOT, 'bench.py')!r}, run_name='__main__')\n"
        "loaded = sorted(m for m in sys.modules if m.startswith('o_o_solver_b200'))\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'modules': loaded, 'library': 'liboosgpu' in maps}))\n"
    )
    out = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, cwd=ROOT, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    result = json.loads(lines[-2])
    assert result["impl"] == "reference" and result["value"] > 0 and result["config"]["equations"] == 60600
    isolation = json.loads(lines[-1])
    assert isolation == {"modules": [], "library": False}


def test_library_same_shapes_takes_the_large_fronts_of_the_symbolic_structure():
    """The library comparison's fronts: column counts from the node partition and rows from the symbolic structure
    give back the structure's panel values, and the fronts taken are the large ones with rows below (r > 0)."""
    import types

    import numpy as np
    import torch

    from o_o_solver_b200 import SymbolicFactor

    model, fixture, _, _ = bench.load_workload("plate100")
    symbolic = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, fixture["node_order"],
                                             fixture["first_position"], fixture["parent"])
    row_start, _ = symbolic.row_structure()
    r = np.diff(row_start)
    before = np.concatenate([[0], np.cumsum(np.asarray(model.weights)[fixture["node_order"]])])
    first = np.asarray(fixture["first_position"])
    c = before[first[1:]] - before[first[:-1]]
    assert int((c * (c + r)).sum()) == symbolic.panel_value_count

    class Event:
        def __init__(self, **_):
            self.at = 0.0

        def record(self):
            import time
            self.at = time.perf_counter()

        def elapsed_time(self, other):
            return max((other.at - self.at) * 1e3, 1e-6)

    host_torch = types.SimpleNamespace(randn=torch.randn, float64=torch.float64, bmm=torch.bmm,
                                       cuda=types.SimpleNamespace(Event=Event, synchronize=lambda: None,
                                                                  empty_cache=lambda: None))
    result = bench.library_same_shapes(host_torch, "cpu", symbolic, model.weights, fixture)
    large = (c + r > 128) & (r > 0)
    assert result["fronts"] == int(large.sum())
    assert result["shapes"] == len(set(zip(r[large].tolist(), c[large].tolist())))
    assert result["ms"] > 0 and result["tflops"] > 0
    symbolic.close()
