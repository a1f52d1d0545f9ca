"""Multi-rank host logic on CPU: two gloo ranks split a Cornell frame's
sample range, render their parts with the CPU restatement of the path and
reduce the framebuffers; the sum equals one rank rendering the whole range
(up to FP32 summation order).  Also the job assignment used for batches."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]

import oracle  # noqa: E402
from wfpt import shard  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, total):
    sys.path[:0] = [str(ROOT / "wavefront-path-tracer_b200"), str(ROOT / "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    import oracle
    import wfpt
    from wfpt import scenes, shard
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        scene, cam = scenes.cornell_box(24, 24)
        cfg = wfpt.render_config(24, 24, max_depth=6, rr_start_depth=3)
        start, count = shard.sample_ranges(total, world, start=40)[rank]
        fb, _ = oracle.PortScene(scene).render(cam, cfg, sample_start=start, sample_count=count)
        t = torch.from_numpy(fb.copy())
        shard.reduce_framebuffer(t, dst=0)
        if rank == 0:
            np.save(os.path.join(out_dir, "reduced.npy"), t.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.skipif(not oracle.port_available(), reason="oracle port not built (make -C oracle port)")
def test_two_rank_sample_split_reduces_to_full_range(tmp_path):
    import torch.multiprocessing as mp
    total, world = 5, 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), total), nprocs=world,
                       start_method="spawn", join=True)
    reduced = np.load(tmp_path / "reduced.npy")
    import wfpt
    from wfpt import scenes
    scene, cam = scenes.cornell_box(24, 24)
    cfg = wfpt.render_config(24, 24, max_depth=6, rr_start_depth=3)
    full, _ = oracle.PortScene(scene).render(cam, cfg, sample_start=40, sample_count=total)
    assert reduced.mean() > 0
    np.testing.assert_allclose(reduced, full, rtol=1e-5, atol=1e-5)


def test_sample_ranges_partition():
    for total in (0, 1, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            parts = shard.sample_ranges(total, world, start=100)
            assert len(parts) == world
            assert sum(n for _, n in parts) == total
            s = 100
            for start, n in parts:
                assert start == s
                s += n
            counts = [n for _, n in parts]
            assert max(counts) - min(counts) <= 1
    with pytest.raises(ValueError):
        shard.sample_ranges(4, 0)
    assert shard.rank_sample_base(3) == 3 << 20


def test_lpt_assign_balances_and_is_deterministic():
    rng = np.random.default_rng(11)
    costs = (rng.integers(64, 513, 64) ** 2 * rng.choice([4, 16, 64], 64)).astype(float)
    owner = shard.lpt_assign(costs, 4)
    assert owner == shard.lpt_assign(list(costs), 4)
    loads = np.bincount(owner, weights=costs, minlength=4)
    # LPT is within 4/3 of the optimum; the optimum is at least the mean load
    assert loads.max() <= 4.0 / 3.0 * max(loads.mean(), costs.max()) + 1e-9
    assert shard.lpt_assign([5.0, 5.0], 2) == [0, 1]
