"""Distributed render jobs: the reference's task layer on one process per GPU.

The reference splits a job into a deterministic table of render tasks,
(tile, sample range) pairs (createRenderTasks, src/distributed/task.cpp:
34-75).  A coordinator hands them to workers over TCP, merges each result
into the job's accumulated radiance and per-pixel sample counts
(DistributedCoordinator::commitResult, src/distributed/coordinator.cpp:
42-90), and periodically writes a checkpoint ("PTDIST1",
src/distributed/checkpoint.cpp) from which it can resume.

Here every rank builds the same task table.  The pending tasks are dealt
round-robin over the ranks, with no messages: task i goes to rank
i mod world.  Each rank renders its tasks through its own Renderer (the task
call, wf_render of the tile and sample range) and merges them as the
coordinator does.  One reduce sums the ranks' contributions onto rank 0
(NCCL between GPUs, gloo on CPU), and one more ORs their completion flags.
Rank 0 then holds the coordinator's state and writes a checkpoint in the
reference's file layout: a job can resume from either side's checkpoint.
Rendering needs no communication; only the merge at the end (or at a
checkpoint) crosses ranks.

Which bytes match the reference: the header, task table, sample counts and
completion flags always do.  The radiance bytes match a reference
coordinator's only for one rank on a fresh job.  The coordinator adds each
task into its running FP32 total as the task arrives; here each rank first
sums its own tasks, the ranks' sums are reduced, and a resumed job adds the
total to the restored radiance, so with several ranks or a resume the FP32
additions are rounded in a different order.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np

TASK_DTYPE = np.dtype([("tile", "<u4"), ("sample_start", "<u4"), ("sample_count", "<u4"), ("x", "<u4"),
                       ("y", "<u4"), ("width", "<u4"), ("height", "<u4")])

_MAGIC = b"PTDIST1\0"
_VERSION = 1
# CheckpointHeader (checkpoint.cpp:10-27): magic, version, header size,
# fingerprint, width, height, tile width, tile height, spp, spp per task,
# sequence, pixel count, task count, payload bytes, payload checksum
_HEADER = struct.Struct("<8sIIQIIIIIIQQQQQ")
assert _HEADER.size == 88
_FNV_OFFSET = 1469598103934665603
_FNV_PRIME = 1099511628211
_MASK64 = (1 << 64) - 1


def create_render_tasks(width, height, tile_width, tile_height, spp, spp_per_task, fingerprint=0):
    """createRenderTasks (task.cpp:34-75): tiles in row-major order, each
    tile's sample ranges in order.  Empty when any size is zero."""
    if not (width and height and tile_width and tile_height and spp and spp_per_task):
        return np.zeros(0, TASK_DTYPE)
    rows = []
    ordinal = 0
    for y in range(0, height, tile_height):
        for x in range(0, width, tile_width):
            w, h = min(tile_width, width - x), min(tile_height, height - y)
            for start in range(0, spp, spp_per_task):
                rows.append((ordinal, start, min(spp_per_task, spp - start), x, y, w, h))
            ordinal += 1
    return np.array(rows, TASK_DTYPE)


def _fnv(data, value=_FNV_OFFSET):
    for byte in data:
        value = ((value ^ byte) * _FNV_PRIME) & _MASK64
    return value


def render_task_key(fingerprint, tile, sample_start, sample_count):
    """computeRenderTaskKey (task.cpp:27-32): FNV-1a over the little-endian
    fingerprint, tile ordinal, sample start and sample count."""
    return _fnv(struct.pack("<QIII", fingerprint & _MASK64, tile, sample_start, sample_count))


@dataclass
class JobConfig:
    """DistributedJobConfig (include/distributed/checkpoint.hpp:9-27)."""
    fingerprint: int
    width: int
    height: int
    tile_width: int
    tile_height: int
    spp: int
    spp_per_task: int

    def tasks(self):
        return create_render_tasks(self.width, self.height, self.tile_width, self.tile_height, self.spp,
                                   self.spp_per_task, self.fingerprint)


@dataclass
class Checkpoint:
    """DistributedCheckpoint (checkpoint.hpp:29-38): unnormalised radiance
    sums (pixels, 3) float32, sample counts (pixels,) uint32, and one
    completion flag per task."""
    job: JobConfig
    sequence: int
    radiance: np.ndarray
    sample_counts: np.ndarray
    completed: np.ndarray


def _validate(c: Checkpoint):
    pixels = c.job.width * c.job.height
    if c.radiance.shape != (pixels, 3) or c.sample_counts.shape != (pixels,):
        raise ValueError("distributed checkpoint pixel buffers have inconsistent sizes")
    if (c.completed > 1).any():
        raise ValueError("distributed checkpoint completion bitmap contains an invalid value")


def write_checkpoint(path, c: Checkpoint):
    """writeDistributedCheckpoint (checkpoint.cpp:67-126): header and payload
    to `path`.tmp, then renamed over `path`."""
    radiance = np.ascontiguousarray(c.radiance, np.float32).reshape(-1, 3)
    counts = np.ascontiguousarray(c.sample_counts, np.uint32).reshape(-1)
    completed = np.ascontiguousarray(c.completed, np.uint8).reshape(-1)
    c = Checkpoint(c.job, c.sequence, radiance, counts, completed)
    _validate(c)
    payload = radiance.nbytes + counts.nbytes + completed.nbytes
    j = c.job
    header = _HEADER.pack(_MAGIC, _VERSION, _HEADER.size, j.fingerprint & _MASK64, j.width, j.height, j.tile_width,
                          j.tile_height, j.spp, j.spp_per_task, c.sequence, len(counts), len(completed), payload,
                          checksum_payload(radiance, counts, completed))
    tmp = str(path) + ".tmp"
    with open(tmp, "wb") as f:
        f.write(header)
        f.write(radiance.tobytes())
        f.write(counts.tobytes())
        f.write(completed.tobytes())
    os.replace(tmp, path)


def checksum_payload(radiance, counts, completed):
    """payloadChecksum (checkpoint.cpp:43-52): one FNV-1a stream over the
    radiance, sample-count and completion bytes (wf_fnv1a64)."""
    from .native import library
    data = np.concatenate([np.ascontiguousarray(radiance, np.float32).view(np.uint8).reshape(-1),
                           np.ascontiguousarray(counts, np.uint32).view(np.uint8).reshape(-1),
                           np.ascontiguousarray(completed, np.uint8).reshape(-1)])
    return int(library().wf_fnv1a64(data.ctypes.data, data.nbytes, 0))


def read_checkpoint(path) -> Checkpoint:
    """readDistributedCheckpoint (checkpoint.cpp:128-216), with its checks:
    magic, version and header size; dimensions; payload size; file size;
    checksum; completion flags."""
    data = open(path, "rb").read()
    if len(data) < _HEADER.size:
        raise ValueError("unsupported or truncated distributed checkpoint header")
    (magic, version, header_size, fingerprint, width, height, tw, th, spp, spt, sequence, pixels, tasks, payload,
     checksum) = _HEADER.unpack_from(data)
    if magic != _MAGIC or version != _VERSION or header_size != _HEADER.size:
        raise ValueError("unsupported or truncated distributed checkpoint header")
    if width * height != pixels or width * height > _MASK64:
        raise ValueError("distributed checkpoint dimensions are invalid")
    if payload != pixels * 12 + pixels * 4 + tasks:
        raise ValueError("distributed checkpoint payload size is invalid")
    if len(data) != _HEADER.size + payload:
        raise ValueError("distributed checkpoint file is truncated or has trailing data")
    at = _HEADER.size
    radiance = np.frombuffer(data, np.float32, pixels * 3, at).reshape(pixels, 3).copy()
    at += pixels * 12
    counts = np.frombuffer(data, np.uint32, pixels, at).copy()
    at += pixels * 4
    completed = np.frombuffer(data, np.uint8, tasks, at).copy()
    if checksum_payload(radiance, counts, completed) != checksum:
        raise ValueError("distributed checkpoint payload checksum does not match")
    c = Checkpoint(JobConfig(fingerprint, width, height, tw, th, spp, spt), sequence, radiance, counts, completed)
    _validate(c)
    return c


class Coordinator:
    """DistributedCoordinator's merge state (coordinator.cpp): the task table,
    accumulated radiance, per-pixel sample counts and completion flags."""

    def __init__(self, job: JobConfig):
        self.job = job
        self.tasks = job.tasks()
        pixels = job.width * job.height
        self.radiance = np.zeros((pixels, 3), np.float32)
        self.sample_counts = np.zeros(pixels, np.uint32)
        self.completed = np.zeros(len(self.tasks), np.uint8)
        self._index = {(int(t["tile"]), int(t["sample_start"]), int(t["sample_count"])): i
                       for i, t in enumerate(self.tasks)}

    def find(self, tile, sample_start, sample_count):
        return self._index.get((tile, sample_start, sample_count))

    def commit(self, task_index, radiance, sample_count=None):
        """commitResult (coordinator.cpp:42-90): adds a task's tile sums.
        Returns "committed", "duplicate" or "rejected"."""
        if task_index is None or not 0 <= task_index < len(self.tasks):
            return "rejected"
        if self.completed[task_index]:
            return "duplicate"
        t = self.tasks[task_index]
        count = int(t["sample_count"]) if sample_count is None else int(sample_count)
        w, h, x, y = int(t["width"]), int(t["height"]), int(t["x"]), int(t["y"])
        radiance = np.asarray(radiance, np.float32)
        if count != int(t["sample_count"]) or radiance.size != w * h * 3:
            return "rejected"
        rows = (np.arange(h)[:, None] + y) * self.job.width + (np.arange(w)[None, :] + x)
        idx = rows.reshape(-1)
        if (self.sample_counts[idx].astype(np.uint64) + count > 0xFFFFFFFF).any():
            return "rejected"
        self.radiance[idx] += radiance.reshape(-1, 3)
        self.sample_counts[idx] += np.uint32(count)
        self.completed[task_index] = 1
        return "committed"

    def restore(self, c: Checkpoint):
        """restore (coordinator.cpp:143-173)."""
        if c.job != self.job:
            raise ValueError("distributed checkpoint job configuration does not match coordinator")
        if len(c.completed) != len(self.tasks) or c.radiance.shape != self.radiance.shape:
            raise ValueError("distributed checkpoint dimensions or task count do not match coordinator")
        self.radiance = c.radiance.copy()
        self.sample_counts = c.sample_counts.copy()
        self.completed = c.completed.copy()

    def snapshot(self, sequence):
        return Checkpoint(self.job, sequence, self.radiance.copy(), self.sample_counts.copy(), self.completed.copy())

    def pending(self):
        return np.nonzero(self.completed == 0)[0]

    def image(self):
        """Mean radiance per pixel, (height, width, 3); zero where no samples."""
        n = np.maximum(self.sample_counts, 1).astype(np.float32)
        return (self.radiance / n[:, None]).reshape(self.job.height, self.job.width, 3)


def assign_tasks(pending, world):
    """Round-robin deal of the pending task indices: rank r renders
    pending[r], pending[r + world], ..."""
    return [np.asarray(pending)[r::world] for r in range(world)]


def run_job(job: JobConfig, render, rank=0, world=1, resume=None, checkpoint_path=None, sequence=None,
            group=None, max_tasks=None):
    """Renders the job's pending tasks over `world` ranks and merges them on
    rank 0.  `render(task)` returns the tile's unnormalised sums (height,
    width, 3) for the task record (the task call of a Renderer,
    render_task((x, y, w, h), sample_start, sample_count)).  `resume` is a
    Checkpoint (or a path) whose completed tasks are skipped; `max_tasks`
    stops each rank after that many tasks (a partial run to checkpoint).
    Rank 0 returns its Coordinator (and writes `checkpoint_path` when given);
    other ranks return None.  With world > 1, torch.distributed must be
    initialised; the three reduces run on every rank in the same order.
    The merged radiance equals a reference coordinator's bit for bit only
    for world == 1 without `resume` (the sums are grouped per rank and added
    to the restored total last, so the FP32 rounding order differs)."""
    coordinator = Coordinator(job)
    base_sequence = 0
    if resume is not None:
        c = read_checkpoint(resume) if isinstance(resume, (str, os.PathLike)) else resume
        coordinator.restore(c)
        base_sequence = c.sequence
    mine = assign_tasks(coordinator.pending(), world)[rank]
    if max_tasks is not None:
        mine = mine[:max_tasks]
    local = Coordinator(job)
    for i in mine:
        t = coordinator.tasks[i]
        local.commit(int(i), render(t))
    if world > 1:
        import torch
        import torch.distributed as dist
        device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        radiance = torch.from_numpy(local.radiance).to(device)
        counts = torch.from_numpy(local.sample_counts.astype(np.int64)).to(device)
        flags = torch.from_numpy(local.completed.astype(np.int32)).to(device)
        dist.reduce(radiance, dst=0, op=dist.ReduceOp.SUM, group=group)
        dist.reduce(counts, dst=0, op=dist.ReduceOp.SUM, group=group)
        dist.reduce(flags, dst=0, op=dist.ReduceOp.MAX, group=group)
        if rank != 0:
            return None
        local.radiance = radiance.cpu().numpy()
        local.sample_counts = counts.cpu().numpy().astype(np.uint32)
        local.completed = flags.cpu().numpy().astype(np.uint8)
    coordinator.radiance += local.radiance
    coordinator.sample_counts += local.sample_counts
    coordinator.completed |= local.completed
    if checkpoint_path is not None:
        write_checkpoint(checkpoint_path, coordinator.snapshot(base_sequence + 1 if sequence is None else sequence))
    return coordinator


def renderer_task_call(renderer):
    """render(task) for run_job from a wfpt.Renderer: the reference's task
    call, a cleared tile rendered over the task's absolute sample range."""
    def render(t):
        return renderer.render_task((int(t["x"]), int(t["y"]), int(t["width"]), int(t["height"])),
                                    int(t["sample_start"]), int(t["sample_count"]))
    return render
