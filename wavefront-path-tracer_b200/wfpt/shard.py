"""Splitting render work over ranks (one process per GPU).

The reference distributes work as tasks over (tile, sample range)
(render_task.cuh:11-29; RenderTaskRenderer::render sums an absolute sample
range of a tile).  Every pixel's samples are independent, so ranks need no
exchange while they render: each holds a read-only scene replica, renders its
own absolute sample range of the frame, and the framebuffers are summed once
at the end (or at a checkpoint) with one reduce.
"""

RANK_SAMPLE_STRIDE = 1 << 20  # absolute sample-index base of rank r in weak scaling


def rank_sample_base(rank):
    """Absolute first sample of `rank` when every rank renders its own
    stream of samples (weak scaling: per-rank work fixed as ranks grow)."""
    return int(rank) * RANK_SAMPLE_STRIDE


def sample_ranges(total, world, start=0):
    """Contiguous split of the sample range [start, start + total) into
    `world` parts (strong scaling); the first total % world ranks get one
    more sample.  Returns [(sample_start, sample_count), ...]."""
    if world <= 0:
        raise ValueError("world size must be positive")
    if total < 0:
        raise ValueError("sample count must be non-negative")
    base, extra = divmod(int(total), int(world))
    out, s = [], int(start)
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((s, n))
        s += n
    return out


def lpt_assign(costs, world):
    """Longest-processing-time-first assignment of independent render jobs
    (cost estimates, e.g. pixels * spp * log2(triangles)) to `world` ranks.
    Ties go to the lower job index and the lower rank, so every rank computes
    the same plan.  Returns the rank of each job."""
    if world <= 0:
        raise ValueError("world size must be positive")
    order = sorted(range(len(costs)), key=lambda j: (-float(costs[j]), j))
    load = [0.0] * world
    owner = [0] * len(costs)
    for j in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[j] = r
        load[r] += float(costs[j])
    return owner


def reduce_framebuffer(framebuffer, dst=0, group=None):
    """Sums the ranks' framebuffers (a torch tensor) into `dst` in place with
    one collective (NCCL on GPUs, gloo on CPU)."""
    import torch.distributed as dist
    dist.reduce(framebuffer, dst=dst, op=dist.ReduceOp.SUM, group=group)
    return framebuffer
