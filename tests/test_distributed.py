"""Distributed render jobs (wfpt.distributed) against the reference's task
layer, compiled into oracle/_ref/libwfref_det.so from src/distributed/
task.cpp and checkpoint.cpp: the same deterministic task table and task
keys, checkpoint files each side reads from the other (byte-identical for
the same state), the reader's rejections, the coordinator's merge rules, and
two gloo ranks splitting a job, checkpointing part of it and resuming."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from wfpt import distributed as wd

ROOT = Path(__file__).resolve().parents[1]
needs_oracle = pytest.mark.skipif(not oracle.available(det=True), reason="oracle/_ref/libwfref_det.so not built")
SHAPES = [(64, 48, 16, 16, 8, 4), (70, 33, 16, 10, 7, 3), (5, 5, 8, 8, 1, 4), (128, 1, 64, 1, 32, 32),
          (0, 10, 4, 4, 1, 1), (10, 10, 4, 4, 0, 1)]


@needs_oracle
@pytest.mark.parametrize("shape", SHAPES)
def test_task_table_matches_the_reference(shape):
    ours = wd.create_render_tasks(*shape, fingerprint=0x1234)
    theirs = oracle.dist_tasks(*shape, fingerprint=0x1234)
    assert len(ours) == len(theirs)
    if len(ours):
        assert np.array_equal(ours.view(np.uint32).reshape(-1, 7), theirs)


@needs_oracle
def test_task_keys_match_the_reference():
    rng = np.random.default_rng(3)
    for _ in range(50):
        fp = int(rng.integers(0, 2**63)) * 2 + int(rng.integers(0, 2))
        tile, start, count = (int(x) for x in rng.integers(0, 2**32, 3, dtype=np.uint64))
        assert wd.render_task_key(fp, tile, start, count) == oracle.dist_task_key(fp, tile, start, count)


def _state(job, seed):
    rng = np.random.default_rng(seed)
    pixels = job.width * job.height
    n = len(job.tasks())
    return (rng.standard_normal((pixels, 3)).astype(np.float32), rng.integers(0, 64, pixels).astype(np.uint32),
            (rng.random(n) < 0.5).astype(np.uint8))


@needs_oracle
def test_checkpoints_are_read_by_either_side_and_identical(tmp_path):
    job = wd.JobConfig(0xDEADBEEFCAFEF00D, 37, 21, 16, 8, 12, 5)
    radiance, counts, completed = _state(job, 1)
    ours, theirs = tmp_path / "ours.ckpt", tmp_path / "theirs.ckpt"
    wd.write_checkpoint(ours, wd.Checkpoint(job, 7, radiance, counts, completed))
    oracle.dist_checkpoint_write(theirs, job.fingerprint, (37, 21, 16, 8, 12, 5), 7, radiance, counts, completed)
    assert ours.read_bytes() == theirs.read_bytes()
    header, r, c, k = oracle.dist_checkpoint_read(ours)
    assert header.tolist() == [job.fingerprint, 37, 21, 16, 8, 12, 5, 7, len(completed)]
    assert np.array_equal(r.view(np.uint32), radiance.view(np.uint32)) and np.array_equal(c, counts)
    assert np.array_equal(k, completed)
    back = wd.read_checkpoint(theirs)
    assert back.job == job and back.sequence == 7 and np.array_equal(back.completed, completed)
    assert np.array_equal(back.radiance.view(np.uint32), radiance.view(np.uint32))


@needs_oracle
@pytest.mark.parametrize("spoil", ["truncated", "trailing", "magic", "checksum", "flag", "header"])
def test_checkpoint_rejections_match_the_reference(tmp_path, spoil):
    job = wd.JobConfig(99, 8, 4, 4, 4, 4, 2)
    radiance, counts, completed = _state(job, 2)
    path = tmp_path / "c.ckpt"
    wd.write_checkpoint(path, wd.Checkpoint(job, 1, radiance, counts, completed))
    data = bytearray(path.read_bytes())
    if spoil == "truncated":
        data = data[:-3]
    elif spoil == "trailing":
        data += b"\0"
    elif spoil == "magic":
        data[6] = ord("2")
    elif spoil == "checksum":
        data[100] ^= 1
    elif spoil == "flag":
        # a completion flag of 2 with a checksum that matches it
        data[-1] = 2
        payload = np.frombuffer(bytes(data[88:]), np.uint8)
        from wfpt.native import library
        data[80:88] = int(library().wf_fnv1a64(payload.ctypes.data, payload.nbytes, 0)).to_bytes(8, "little")
    else:
        data = data[:40]
    path.write_bytes(bytes(data))
    with pytest.raises(ValueError) as ours:
        wd.read_checkpoint(path)
    with pytest.raises(ValueError) as theirs:
        oracle.dist_checkpoint_read(path)
    assert str(ours.value) == str(theirs.value)


def test_coordinator_merge_rules():
    job = wd.JobConfig(5, 6, 4, 4, 4, 3, 2)
    co = wd.Coordinator(job)
    assert len(co.tasks) == 4  # two tiles x two sample ranges (2 + 1)
    t = co.tasks[1]
    assert (int(t["sample_start"]), int(t["sample_count"])) == (2, 1)
    tile = np.ones((4, 4, 3), np.float32)
    assert co.commit(0, tile) == "committed"
    assert co.commit(0, tile) == "duplicate"
    assert co.commit(1, tile, sample_count=2) == "rejected"
    assert co.commit(9, tile) == "rejected"
    assert co.commit(2, np.ones((4, 2, 3), np.float32)) == "committed"  # the ragged second tile
    assert co.sample_counts.reshape(4, 6)[0].tolist() == [2, 2, 2, 2, 2, 2]
    assert co.pending().tolist() == [1, 3]
    other = wd.Coordinator(job)
    other.restore(co.snapshot(3))
    assert np.array_equal(other.radiance, co.radiance) and other.pending().tolist() == [1, 3]
    with pytest.raises(ValueError):
        wd.Coordinator(wd.JobConfig(6, 6, 4, 4, 4, 3, 2)).restore(co.snapshot(3))


def _fake_render(t):
    # deterministic, exactly representable tile sums: (tile + 1) * samples
    v = np.float32((int(t["tile"]) + 1) * int(t["sample_count"]))
    return np.full((int(t["height"]), int(t["width"]), 3), v, np.float32)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, partial):
    sys.path[:0] = [str(ROOT / "wavefront-path-tracer_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    from wfpt import distributed as wd
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        job = wd.JobConfig(77, 40, 30, 16, 16, 10, 4)
        path = os.path.join(out_dir, "job.ckpt")
        if partial:
            wd.run_job(job, _fake_render, rank, world, checkpoint_path=path, max_tasks=2)
        else:
            wd.run_job(job, _fake_render, rank, world, resume=path, checkpoint_path=path + ".final")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_checkpoint_and_resume(tmp_path):
    import torch.multiprocessing as mp
    for partial in (True, False):
        mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), partial), nprocs=2, join=True,
                           start_method="spawn")
    job = wd.JobConfig(77, 40, 30, 16, 16, 10, 4)
    first = wd.read_checkpoint(tmp_path / "job.ckpt")
    assert first.sequence == 1 and int(first.completed.sum()) == 4  # two tasks on each rank
    final = wd.read_checkpoint(tmp_path / "job.ckpt.final")
    assert final.sequence == 2 and final.completed.all()
    whole = wd.run_job(job, _fake_render)  # one rank, every task
    assert np.array_equal(final.radiance, whole.radiance)
    assert np.array_equal(final.sample_counts, whole.sample_counts)
    assert (final.sample_counts == 10).all()
