"""Generates the golden fixtures of the tests and the benchmark from the reference itself (oracle/_ref/liboos_ref.so,
built from the reference's sources by oracle/Makefile). Run in a container that has the reference:

    make -C oracle REF=/path/to/O_o_Solver && python tests/golden/make_golden.py

Writes, for each workload of the benchmark and the tests:
  orderings/<name>.npz   the reference's final node order (ConstrainedOrdering, then SymbolicFactor::analyse's
                         postorder) and its supernode partition (first positions, parents): the symbolic stage the
                         reference computes, reused as it is by the GPU path (the row structures follow from them);
  solutions/<name>.npz   for small cases: the reference's inertia, pivot diagnostics and solutions of seeded
                         right-hand sides (the known answers the GPU path is checked against on the GPU box, where the
                         reference is not built);
  modes/<name>.npz       the reference's lowest modes of a pencil (SparsePencil + BlockLanczos::solve, block 8): the
                         eigenvalues, the shifts with their Sturm counts, the factorisations.

    python tests/golden/make_golden.py [--modes-only] [--with-large-modes] [--only=name,name,...]
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

ORDERINGS = {
    # name: (kind, size)
    "plate6": ("plate", 6),
    "plate20": ("plate", 20),
    "plate100": ("plate", 100),
    "plate200": ("plate", 200),
    "plate580": ("plate", 580),
    "hex4": ("hex", 4),
    "hex8": ("hex", 8),
    "hex14": ("hex", 14),
    "hex30": ("hex", 30),
    "hex60": ("hex", 60),
    # the batched stiffened panels: one skin topology per mesh size (the blades add no adjacency)
    **{f"panel{m}": ("panel", m) for m in (18, 22, 26, 30, 34, 38, 42, 46, 50, 55, 60, 65, 70, 75, 78, 81)},
    # the wing box of the learned start (one topology; the design variables change values only)
    "wingbox": ("wingbox", 0),
    # a small wing box for the tests of the learned start
    "wingbox_small": ("wingbox", 1),
}
SOLUTIONS = ["plate6", "plate20", "hex4", "hex8"]
# name: (modes, block size); the large ones (minutes on a few cores) only with --with-large-modes.
MODES = {"hex8": (20, 8), "hex14": (20, 8), "plate20": (12, 7), "hex30": (20, 8)}
LARGE_MODES = {"hex60": (20, 8)}


def pencil_of(kind, model, sym):
    """K and M in the reference's order: the hex's lumped mass, or for a plate the translations of a 2 mm aluminium
    sheet without rotary inertia (a mass with a null space)."""
    from o_o_solver_b200 import SymmetricCsc

    k = model.csc(sym.node_order, 0)
    if kind == "hex":
        return k, model.csc(sym.node_order, 1)
    size = model.spec.nx
    values = np.zeros_like(k.values)
    mass = np.zeros(sym.dof_count)
    mass[np.arange(sym.dof_count) % 6 < 3] = 2700.0 * 0.002 / (size * size)
    values[k.offsets[:-1]] = mass
    return k, SymmetricCsc(k.offsets, k.rows, values)


def make_modes(names, threads):
    import oracle

    os.makedirs(os.path.join(HERE, "modes"), exist_ok=True)
    for name, (count, block) in names.items():
        kind, size = ORDERINGS[name]
        model = model_of(kind, size)
        sym = oracle.analyse(model.offsets, model.neighbours, model.weights, model.coordinates, threads=threads)
        k, m = pencil_of(kind, model, sym)
        result = oracle.modes(sym, k.offsets, k.rows, k.values, m.values, count, block_size=block, threads=threads,
                              vectors=False)
        np.savez_compressed(os.path.join(HERE, "modes", name + ".npz"), eigenvalues=result["eigenvalues"],
                            shifts=result["shifts"], factorisations=np.array(result["factorisations"]),
                            verified=np.array(result["verified"]), block_size=np.array(block),
                            seconds=np.array(result["seconds"]), threads=np.array(threads))
        print(f"{name}: {count} modes in {result['seconds']:.1f} s on {threads} threads, "
              f"{result['factorisations']} factorisations, lowest {result['eigenvalues'][0]:.6e}")


def wing_box_spec(thicknesses, small=False):
    """The wing box of the learned start (span 10 m, chord 2 m, height 0.3 m, ribs every 0.5 m, shells of 0.05 m), or
    the small one of its tests (span 2 m, chord 0.6 m, height 0.15 m)."""
    from o_o_solver_b200 import workloads

    if small:
        return workloads.WingBoxSpec(thicknesses=tuple(thicknesses), span=2.0, chord=0.6, height=0.15)
    return workloads.WingBoxSpec(thicknesses=tuple(thicknesses))


def model_of(kind, size):
    from o_o_solver_b200 import workloads

    if kind == "plate":
        return workloads.Model(workloads.PlateSpec(size, size))
    if kind == "panel":
        return workloads.Model(workloads.PlateSpec(size, size, 0.5, 0.5))
    if kind == "wingbox":
        return workloads.Model(wing_box_spec((0.002,) * 24, small=size == 1))
    return workloads.Model(workloads.HexSpec(size))


def main():
    import oracle

    threads = os.cpu_count() or 1
    if "--modes-only" not in sys.argv:
        make_orderings(threads)
    if any(a.startswith("--only=") for a in sys.argv):
        return
    make_modes(MODES, threads)
    if "--with-large-modes" in sys.argv:
        make_modes(LARGE_MODES, threads)


def make_orderings(threads):
    import oracle

    os.makedirs(os.path.join(HERE, "orderings"), exist_ok=True)
    os.makedirs(os.path.join(HERE, "solutions"), exist_ok=True)
    only = next((a.split("=", 1)[1].split(",") for a in sys.argv if a.startswith("--only=")), None)
    for name, (kind, size) in ORDERINGS.items():
        if only is not None and name not in only:
            continue
        model = model_of(kind, size)
        sym = oracle.analyse(model.offsets, model.neighbours, model.weights, model.coordinates, threads=threads)
        np.savez_compressed(os.path.join(HERE, "orderings", name + ".npz"), node_order=sym.node_order,
                            first_position=sym.first_position, parent=sym.parent, flops=np.array(sym.flops),
                            dof_count=np.array(sym.dof_count), supernode_count=np.array(sym.supernode_count))
        print(f"{name}: {sym.dof_count} DOFs, {sym.supernode_count} supernodes, {sym.flops:.3e} flops")
        if name not in SOLUTIONS:
            continue
        csc = model.csc(sym.node_order)
        factor = oracle.factorise(sym, csc.offsets, csc.rows, csc.values, family=0)
        rng = np.random.default_rng(20261203)
        b = np.asfortranarray(rng.standard_normal((sym.dof_count, 3)))
        x = factor.solve(b)
        np.savez_compressed(os.path.join(HERE, "solutions", name + ".npz"), b=b, x=x,
                            inertia=np.array([factor.positive, factor.negative, factor.zero]),
                            issue_count=np.array(factor.issue_count),
                            equation_of_largest=np.array(factor.equation_of_largest),
                            largest_ratio=np.array(factor.largest_ratio))


if __name__ == "__main__":
    main()
