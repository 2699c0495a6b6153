"""The batched form's host side (CPU): the block-diagonal join of several models is exactly the block diagonal of their
matrices, its symbolic structure is the models' structures side by side, and the seeded panel cases are reproducible
and span the stated sizes."""

import os

import numpy as np
import scipy.sparse as sp

from o_o_solver_b200 import batch, workloads

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orderings")


def fixture_of(n):
    return dict(np.load(os.path.join(GOLDEN, f"panel{n}.npz")))


def lower(csc, n):
    return sp.csc_matrix((csc.values, csc.rows, csc.offsets), shape=(n, n))


def test_join_is_the_block_diagonal(lib):
    cases = [batch.PanelCase(18, 4, 0.001), batch.PanelCase(22, 7, 0.003), batch.PanelCase(18, 12, 0.002)]
    joined, rhs, parts = batch.panel_batch(cases, fixture_of, columns=3)
    n = joined.dimension
    assert n == sum(p.dof_count for p in parts)
    blocks = [lower(p.matrix, p.dof_count) for p in parts]
    assert abs(lower(joined.matrix, n) - sp.block_diag(blocks)).max() == 0.0
    # the symbolic structure: every supernode's rows inside its own model
    row_start, rows = joined.symbolic.row_structure()
    assert joined.symbolic.supernode_count == sum(len(p.parent) for p in parts)
    assert joined.symbolic.flop_count > 0
    for i in range(len(parts)):
        lo, hi = joined.dof_offsets[i], joined.dof_offsets[i + 1]
        part_rows = rows[(rows >= lo) & (rows < hi)]
        assert len(part_rows) == len(parts[i].rows)
    # the loads: each model's own, stacked
    for i, b in enumerate(joined.split(rhs)):
        assert b.shape == (parts[i].dof_count, 3)
        assert np.linalg.norm(b[:, 0]) > 0


def test_panel_cases_are_seeded():
    a = batch.panel_cases(64)
    b = batch.panel_cases(64)
    assert a == b
    assert {c.n for c in a} <= set(batch.PANEL_SIZES)
    assert all(4 <= c.stringers <= 12 and 0.001 <= c.thickness <= 0.004 for c in a)
    assert batch.panel_cases(64, seed=1) != a


def test_blades_stiffen_the_skin(lib):
    order = np.arange(18 * 19, dtype=np.int32)
    skin = workloads.Model(workloads.PlateSpec(18, 18, 0.5, 0.5))
    panel = workloads.Model(workloads.PanelSpec(n=18, stringers=4))
    skin_csc, panel_csc = skin.csc(order), panel.csc(order)
    # the same stored pattern (the blades lie on the skin's grid lines), more stiffness on the blades' nodes
    assert np.array_equal(skin_csc.offsets, panel_csc.offsets) and np.array_equal(skin_csc.rows, panel_csc.rows)
    k_skin = lower(skin_csc, skin.dof_count).toarray()
    k_panel = lower(panel_csc, panel.dof_count).toarray()
    assert np.all(np.diag(k_panel) >= np.diag(k_skin) - 1e-9 * np.abs(np.diag(k_skin)))
    assert np.diag(k_panel).sum() > np.diag(k_skin).sum()


def test_deal_covers_every_panel_once_and_balances():
    rng = np.random.default_rng(4)
    work = rng.uniform(1, 100, 97)
    for ranks in (1, 2, 3, 8):
        shares = batch.deal(work, ranks)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(97))
        loads = [work[s].sum() for s in shares]
        assert max(loads) - min(loads) <= work.max()


def _deal_rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cases = batch.panel_cases(40)
    flops = [float(np.load(os.path.join(GOLDEN, f"panel{c.n}.npz"))["flops"]) for c in cases]
    mine = batch.deal(flops, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    out.put((rank, gathered))
    dist.destroy_process_group()


def test_deal_agrees_across_two_gloo_ranks():
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_deal_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert results[0] == results[1]
    shares = results[0]
    assert sorted(shares[0] + shares[1]) == list(range(40)) and not set(shares[0]) & set(shares[1])
