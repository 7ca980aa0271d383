"""Replica plumbing on real localization rows: two gloo ranks, each with its own
context on cuda:0, run the frame pipeline on their contiguous shares of a
stack (frames numbered from their share's start) and rank 0 gathers the rows;
they equal one process's rows over the whole stack, ids renumbered.  The two
ranks' kernels never wait on one another; only host bookkeeping crosses
ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

S, R, NF = 96, 16, 7


def _stack():
    import oracle as O
    from common import OPTICS, astig_zernike
    from test_gpu_detect import make_frames
    ref = O.OraclePSF(64, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, astig_zernike())
    return make_frames(ref.model, S, NF, seed=314, emitters=4, R=32)


def _localizer(z, ctx):
    from common import OPTICS, astig_zernike
    psf_det = z.PSF(ctx, z.optics(size_fft=64, kz_reset=True, **OPTICS), astig_zernike())
    psf_fit = z.PSF(ctx, z.optics(size_fft=64, **OPTICS), astig_zernike())
    det = z.Detector(psf_det, S, S, R, -0.6, 0.6, 0.11, 0.1)

    def run(frames, frame0=0):
        return z.localize_frames(ctx, det, psf_fit, frames, -0.6, 0.6, photon_threshold=300.0, precision=1,
                                 max_iter=40, frame0=frame0)
    return run, (det, psf_det, psf_fit)


def _worker(rank, world, port, out_path, root):
    import sys
    sys.path[:0] = [root, os.path.join(root, "tests")]
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        import __graft_entry__ as ge
        z = ge.load_package()
        import zola3d_b200.replicas as rp
        ctx = z.Context(0)
        run, objs = _localizer(z, ctx)
        rows = rp.localize_frames_replicated(run, _stack(), rank, world)
        rp.barrier()
        if rank == 0:
            np.save(out_path, rows)
        else:
            assert rows is None
        for o in objs:
            o.close()
        ctx.close()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_replicas_give_the_rows_of_one_process(zpkg, ctx, tmp_path):
    out = str(tmp_path / "rows.npy")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    mp.start_processes(_worker, args=(2, _free_port(), out, root), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    run, objs = _localizer(zpkg, ctx)
    want = run(_stack())
    for o in objs:
        o.close()
    assert len(want) >= 5
    assert got.dtype == want.dtype
    assert np.array_equal(got, want)  # frame order, frames numbered over the stack, ids renumbered
