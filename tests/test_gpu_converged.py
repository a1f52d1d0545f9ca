"""Equal image RMSE against a converged image of the reference's own CUDA
renderer (oracle/converged_oracle.py): the Cornell box, 256x256, depth 8,
Russian roulette from bounce 3.  The converged image here is 4,096 spp
accumulated in FP64 (the measurement itself uses 65,536); at 4, 16 and 64
spp on the same sample ranges both renderers' relative RMSE against it must
agree within 2 % of each other -- they trace the same paths, so only FP32
rounding separates them -- and fall as 1 / sqrt(spp)."""
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB = ROOT / "oracle" / "_ref" / "libwfref_cuda.so"

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not LIB.exists(), reason="reference CUDA build absent (make -C oracle cuda)")]


def test_equal_rmse_against_converged_reference(cuda):
    import converged_oracle
    res = converged_oracle.run("cornell", oracle_spp=4096, levels=(4, 16, 64))
    rows = {row["spp"]: row for row in res["rmse"]}
    for spp, row in rows.items():
        assert abs(row["this_renderer"] - row["reference_cuda"]) <= 0.02 * row["reference_cuda"], row
        assert row["between_renderers"] < 0.1 * row["reference_cuda"], row
    assert 0.4 < rows[16]["this_renderer"] / rows[4]["this_renderer"] < 0.6
    assert 0.18 < rows[64]["this_renderer"] / rows[4]["this_renderer"] < 0.32
