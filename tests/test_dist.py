"""Multi-process host logic on the CPU: row shards by nonzeros cover the
matrix, and with two gloo ranks each rank's y block (computed here by the
oracle, standing in for the device kernel) gathers into the full y; the
timing rule takes the slowest rank."""
import os
import socket

import numpy as np
import pytest

from sciwasm.sparse_b200 import dist, synth


def test_shards_cover_rows_and_balance():
    rp, col, val = synth.power_law(5000, seed=1, cap=300)
    lens = np.diff(rp)
    for world in (1, 2, 3, 8):
        s, e = dist.shard_rows(rp, world)
        assert s[0] == 0 and e[-1] == 5000
        assert np.all(s[1:] == e[:-1]) and np.all(e >= s)
        loads = [int(rp[b] - rp[a]) for a, b in zip(s, e)]
        assert sum(loads) == col.size
        assert max(loads) <= col.size // world + int(lens.max())
        blocks = [dist.local_block(rp, col, val, a, b) for a, b in zip(s, e)]
        assert np.array_equal(np.concatenate([b[1] for b in blocks]), col)
        assert np.array_equal(np.concatenate([b[2] for b in blocks]), val)


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as tdist
    from oracle import binding as orc
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rp, col, val = synth.power_law(4000, seed=2, cap=200)
        x = synth.uniform_vec(4000, 3)
        s, e = dist.shard_rows(rp, world)
        brp, bcol, bval = dist.local_block(rp, col, val, int(s[rank]), int(e[rank]))
        y_local = orc.spmv_csr(brp, bcol, bval, x, np.zeros(brp.size - 1))
        y = dist.gather_rows(torch.from_numpy(y_local), s, e).numpy()
        t = dist.max_over_ranks(1.5 + rank)
        # the padded in-place layout: this rank's block written in place,
        # one all-gather, the padding dropped
        sy = dist.ShardedY(s, e, rank, torch.float64, "cpu")
        sy.local().copy_(torch.from_numpy(y_local))
        sy.allgather()
        q.put((rank, y, t, sy.full().numpy(), sy.gather_bytes(), sy.counts))
    finally:
        tdist.destroy_process_group()


def test_two_gloo_ranks_gather_rows(oracle):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rp, col, val = synth.power_law(4000, seed=2, cap=200)
    x = synth.uniform_vec(4000, 3)
    full = oracle.spmv_csr(rp, col, val, x, np.zeros(4000))
    for rank, y, t, y_padded, nbytes, counts in out:
        assert np.array_equal(y, full)  # each row is computed by one rank
        assert t == 2.5
        assert np.array_equal(y_padded, full)
        assert counts[0] != counts[1]  # ragged blocks (balanced by nonzeros)
        assert nbytes == max(counts) * 8


def test_peer_y_single_rank_layout():
    """PeerY with one rank: its own full-length buffer is the only
    destination, row r starts r values in, and the barrier is a no-op."""
    import torch
    py = dist.PeerY(1000, torch.float64, "cpu")
    assert py.world == 1 and py.ptrs == [py.buf.data_ptr()]
    assert py.rows_ptr(5) == py.buf.data_ptr() + 40
    assert py.ptrs_dev.tolist() == py.ptrs
    py.barrier()
