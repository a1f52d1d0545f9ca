"""The single-scene autotuner (wf_renderer_autotune, wfpt.autotune): every
candidate schedule renders the same sums, so whichever it picks must give
the bit-identical image of the default config; the table covers every
candidate in the tuner's order, and a second call with the same key returns
the cached choice without rendering."""
import numpy as np
import pytest

import wfpt
from wfpt import abi, scenes

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_schedule_with_identical_sums(cuda, tmp_path):
    scene, cam = scenes.cornell_box(64, 64)
    base = wfpt.render_config(64, 64, max_depth=8, rr_start_depth=3)
    dev = wfpt.DeviceScene(scene)
    cache = tmp_path / "tuned.json"
    best, table = wfpt.autotune(dev, cam, base, modes=(abi.MODE_GRAPH, abi.MODE_STREAM, abi.MODE_PERSISTENT),
                                block_sizes=(128, 256), refill_thresholds=(8, 16), concurrent_tiles=(1, 2),
                                regenerate_percents=(10, 50), chunks=(32, 64),
                                persistent_stages=(abi.PERSISTENT_FUSED, abi.PERSISTENT_STAGED), samples=2,
                                key="cornell64", cache_path=str(cache))
    # graph: 2 x 2 x 2 wavefronts, stream: 2 x 2 x 2 percents,
    # persistent: 2 x 2 x (fused x 2 chunks + staged)
    assert len(table) == 28 and all(ms > 0 for _, ms in table)
    fastest = min(table, key=lambda row: row[1])[0]
    assert best.mode == fastest["mode"] and best.block_size == fastest["block_size"]
    again, empty = wfpt.autotune(dev, cam, base, key="cornell64", cache_path=str(cache))
    assert empty == [] and bytes(again) == bytes(best)
    images = []
    for cfg in (base, best):
        r = wfpt.Renderer(dev, cam, cfg)
        images.append(r.render_task((0, 0, 64, 64), 77, 4))
        r.close()
    dev.close()
    assert np.array_equal(images[0].view(np.uint32), images[1].view(np.uint32))
