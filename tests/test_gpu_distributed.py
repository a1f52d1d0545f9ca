"""A distributed render job on the GPU (wfpt.distributed.run_job with the
renderer's task call) against the reference: every task of the job rendered
by the host-compiled reference's own task path and merged in the same order
gives the same accumulated radiance bit for bit, the same sample counts and
completion flags; a job checkpointed part way and resumed ends in the same
state."""
import numpy as np
import pytest

import oracle
import wfpt
from wfpt import distributed as wd
from wfpt import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_oracle():
    if not oracle.available(det=True):
        pytest.skip("oracle/_ref/libwfref_det.so not built")


def test_job_matches_the_reference_task_by_task(tmp_path):
    scene, cam = scenes.cornell_box(48, 40)
    cfg = wfpt.render_config(48, 40, max_depth=6, rr_start_depth=3)
    job = wd.JobConfig(0xC0FFEE, 48, 40, 16, 16, 6, 4)
    dev = wfpt.DeviceScene(scene)
    r = wfpt.Renderer(dev, cam, cfg)
    try:
        render = wd.renderer_task_call(r)
        half = wd.run_job(job, render, checkpoint_path=tmp_path / "half.ckpt", max_tasks=5)
        assert int(half.completed.sum()) == 5
        done = wd.run_job(job, render, resume=tmp_path / "half.ckpt", checkpoint_path=tmp_path / "done.ckpt")
    finally:
        r.close()
        dev.close()
    ref = oracle.RefScene(scene, det=True)
    want = wd.Coordinator(job)
    for i, t in enumerate(want.tasks[:5]):
        tile = (int(t["x"]), int(t["y"]), int(t["width"]), int(t["height"]))
        sums, _, _ = ref.render(cam, cfg, tile=tile, sample_start=int(t["sample_start"]),
                                sample_count=int(t["sample_count"]))
        want.commit(i, sums)
    first_five = want.snapshot(1)
    ref.close()
    assert np.array_equal(half.radiance.view(np.uint32), first_five.radiance.view(np.uint32))
    # the resumed run merges the remaining tasks into a fresh sum, then adds
    # it onto the restored one
    rest = wd.Coordinator(job)
    ref = oracle.RefScene(scene, det=True)
    for i, t in enumerate(rest.tasks):
        if i < 5:
            continue
        tile = (int(t["x"]), int(t["y"]), int(t["width"]), int(t["height"]))
        sums, _, _ = ref.render(cam, cfg, tile=tile, sample_start=int(t["sample_start"]),
                                sample_count=int(t["sample_count"]))
        rest.commit(i, sums)
    ref.close()
    expected = first_five.radiance + rest.radiance
    final = wd.read_checkpoint(tmp_path / "done.ckpt")
    assert final.sequence == 2 and final.completed.all() and (final.sample_counts == 6).all()
    assert np.array_equal(final.radiance.view(np.uint32), expected.view(np.uint32))
    assert np.array_equal(done.radiance.view(np.uint32), expected.view(np.uint32))
