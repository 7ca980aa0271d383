"""CPU tests of the multi-GPU replica plumbing (two gloo ranks on 127.0.0.1)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

DT = np.dtype([("id", np.int32), ("frame", np.int32), ("x_nm", np.float64)])


def _replicas():
    import __graft_entry__ as ge
    ge.load_package()
    import zola3d_b200.replicas as rp
    return rp


def fake_localize(frames, frame0=0):
    """Stand-in for localize_frames: frame f yields (f % 3) rows, ids numbered per call."""
    rows = []
    for k in range(len(frames)):
        f = frame0 + k
        for j in range(f % 3):
            rows.append((len(rows), f, 1000.0 * f + j))
    return np.array(rows, dtype=DT)


def _worker(rank, world, port, out_path, nframes):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        rp = _replicas()
        frames = np.zeros((nframes, 4, 4))
        rows = rp.localize_frames_replicated(fake_localize, frames, rank, world)
        tmax = rp.max_over_ranks(10.0 + rank)
        rp.barrier()
        if rank == 0:
            np.savez(out_path, rows=rows, tmax=tmax)
        else:
            assert rows is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_contiguous_share_partitions_in_order():
    rp = _replicas()
    for n in (0, 1, 7, 10, 1001):
        for world in (1, 2, 3, 8):
            spans = [rp.contiguous_share(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        rp.contiguous_share(5, 2, 2)


def test_single_process_is_the_identity():
    rp = _replicas()
    rows = fake_localize(np.zeros((5, 4, 4)))
    assert rp.gather_rows(rows) is rows
    assert rp.max_over_ranks(3.5) == 3.5


@pytest.mark.parametrize("nframes", [9, 1])
def test_two_rank_replicas_match_one_process(tmp_path, nframes):
    out = str(tmp_path / "rows.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out, nframes), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    want = fake_localize(np.zeros((nframes, 4, 4)))
    assert float(got["tmax"]) == 11.0
    rows = got["rows"]
    assert rows.dtype == DT
    assert np.array_equal(rows, want)  # frame order, ids renumbered over the stack
