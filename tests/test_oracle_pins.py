"""Pins the oracle (the reference's own code, host-compiled into
oracle/_ref/libwfref.so, and its deterministic-math twin libwfref_det.so)
against the golden values and known-answer checks of the reference's tests."""
import ctypes
import math

import numpy as np
import pytest

import oracle
import wfpt
from wfpt import abi, scenes

pytestmark = pytest.mark.skipif(not oracle.available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("det", [False, True])
def test_fresnel_golden_values(det):
    f = oracle.ref_lib(det).wfref_dielectric_reflectance
    # tests/material_transport_tests.cu:119-122
    assert abs(f(1.0, 1 / 1.5) - 0.04) <= 1e-6
    assert abs(f(0.767, 1.5) - 0.23811942) <= 2e-6
    assert f(0.7, 1.5) == 1.0 and f(0.0, 1.0) == 0.0
    # reciprocity, :124-128
    cosine, eta = 0.8, 1 / 1.5
    ct = math.sqrt(1 - eta * eta * (1 - cosine * cosine))
    assert abs(f(cosine, eta) - f(ct, 1 / eta)) <= 1e-6


def test_rng_restatement_matches_reference():
    """A numpy restatement of pixelRngKey/makeRngState/randomFloat
    (rng.cuh:7-51, rng.cu:4-42) agrees with the reference for both strategies."""
    lib = oracle.ref_lib()
    lib.wfref_rng.argtypes = [ctypes.c_uint32] * 4 + [ctypes.c_void_p, ctypes.c_void_p]
    for strategy in (0, 1):
        for pixel, sample in [(0, 0), (1234, 567), (65535, 15), (2073599, 1 << 20)]:
            out = np.zeros(8, np.float32)
            state = ctypes.c_uint64()
            lib.wfref_rng(pixel, sample, strategy, 8, out.ctypes.data, ctypes.addressof(state))
            ours = rng_restatement(pixel, sample, strategy, 8)
            assert np.array_equal(out, ours)


def rng_restatement(pixel, sample, strategy, n):
    M32, M64 = 0xFFFFFFFF, 0xFFFFFFFFFFFFFFFF
    if strategy == 0:
        key = (pixel ^ ((sample * 0x9E3779B9) & M32)) & M32
        seed = (key * 747796405 + 2891336453) & M32
        state = 1 if seed == 0 else seed
    else:
        key = ((sample << 32) | pixel) & M64
        v = (key + 0x9E3779B97F4A7C15) & M64
        v = ((v ^ (v >> 30)) * 0xBF58476D1CE4E5B9) & M64
        v = ((v ^ (v >> 27)) * 0x94D049BB133111EB) & M64
        state = v ^ (v >> 31)
    out = []
    for _ in range(n):
        if strategy == 0:
            x = state
            x ^= (x << 13) & M32
            x ^= x >> 17
            x ^= (x << 5) & M32
            state = x
            value = x
        else:
            old = state
            state = (old * 6364136223846793005 + 1442695040888963407) & M64
            xs = (((old >> 18) ^ old) >> 27) & M32
            rot = old >> 59
            value = ((xs >> rot) | (xs << ((32 - rot) & 31))) & M32
        out.append(np.float32(value >> 8) * np.float32(2.0 ** -24))
    return np.array(out, np.float32)


def test_pcg_seed_uniqueness():
    """rng_tests.cu:14-54: PCG keys of 64x64 pixels x 256 samples never collide."""
    pixel = np.arange(64 * 64, dtype=np.uint64)
    keys = (np.arange(256, dtype=np.uint64)[:, None] << np.uint64(32)) | pixel[None, :]
    with np.errstate(over="ignore"):
        v = keys + np.uint64(0x9E3779B97F4A7C15)
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        v = v ^ (v >> np.uint64(31))
    assert len(np.unique(v)) == v.size


@pytest.mark.parametrize("det", [False, True])
def test_environment_distribution_pins(det):
    """environment_tests.cpp:37-44: constant map normalization."""
    rgba = np.full((8, 16, 4), 8.0, np.float32)
    p, ap, al = oracle.environment_distribution(rgba, det)
    assert abs(p.astype(np.float64).sum() - 1.0) < 1e-6
    assert (ap <= 1.0).all() and (al < p.size).all()
    with pytest.raises(ValueError):
        bad = rgba.copy()
        bad[0, 0, 0] = -1
        oracle.environment_distribution(bad, det)
    # Bright texel: bilinear shoulders receive mass (environment_tests.cpp:66-69).
    rgba = np.zeros((8, 16, 4), np.float32)
    rgba[0, 0, :3] = 10000
    p, _, _ = oracle.environment_distribution(rgba, det)
    assert p[-1] > 0 and p[15] > 0.01 and p[1] > 0.01 and p[16] > 0.01


def test_math_twin_within_one_ulp():
    """libwfref_det.so differs from libwfref.so only by the elementary
    functions, and those agree with the C library within 1 ulp."""
    rng = np.random.RandomState(1)
    x = rng.uniform(-10, 10, 20000).astype(np.float32)
    y = rng.uniform(-10, 10, 20000).astype(np.float32)
    pos = rng.uniform(1e-3, 100, 20000).astype(np.float32)
    unit = rng.uniform(0, 1, 20000).astype(np.float32)
    cases = [(0, x, y), (1, x, y), (2, x * 0.1, y), (3, x, y), (4, pos, y), (5, x * 5, y), (6, unit, np.full_like(x, 5)),
             (7, x, y), (8, x, y)]
    for kind, a, b in cases:
        outs = []
        for det in (False, True):
            lib = oracle.ref_lib(det)
            lib.wfref_math.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
            o = np.zeros(len(a), np.float64)
            lib.wfref_math(kind, a.ctypes.data, b.ctypes.data, len(a), o.ctypes.data)
            outs.append(o)
        if kind >= 7:
            ulp = np.abs(outs[0].view(np.int64) - outs[1].view(np.int64))
        else:
            ulp = np.abs(outs[0].astype(np.float32).view(np.int32).astype(np.int64) -
                         outs[1].astype(np.float32).view(np.int32).astype(np.int64))
        assert ulp.max() <= 1, (kind, ulp.max())


@pytest.mark.parametrize("det", [False, True])
def test_cornell_lights_registered_like_the_reference(det):
    scene, _ = scenes.cornell_box(32, 32)
    ref = oracle.RefScene(scene, det=det)
    rec, alias = ref.lights()
    assert len(rec) == 2
    assert np.allclose(rec[:, 12], 1.125)          # area of each half of the 1.5 x 1.5 quad
    assert np.allclose(rec[:, 14], 0.5)            # selectionPdf
    assert np.allclose(rec[:, 9:12], [0, -1, 0])   # light normals face down
    ref.close()


def test_reference_twins_agree_on_rays():
    """Ray queries involve no elementary functions: both builds agree bit for bit."""
    from helpers import acceleration_rays, hit_diff
    scene, _ = scenes.sphere_field(64, 36, frequency=8)
    rays = acceleration_rays(count=4096)
    a = oracle.RefScene(scene, det=False).trace(rays)
    b = oracle.RefScene(scene, det=True).trace(rays)
    assert len(hit_diff(a, b)) == 0


def test_reference_persistent_equals_graph():
    """The reference's two execution modes produce the same sums and queue counts."""
    scene, cam = scenes.cornell_box(32, 32)
    cfg = wfpt.render_config(32, 32, max_depth=8, rr_start_depth=3)
    ref = oracle.RefScene(scene)
    g, _, cg = ref.render(cam, cfg, sample_count=2)
    p, _, cp = ref.render(cam, cfg, sample_count=2, persistent=True, threads=1)
    assert np.array_equal(g, p) and np.array_equal(cg, cp)


def test_reference_twins_images_close():
    """The math library is the only difference: images agree statistically."""
    from helpers import relative_rmse
    scene, cam = scenes.cornell_box(48, 48)
    cfg = wfpt.render_config(48, 48, max_depth=8, rr_start_depth=3)
    a, _, _ = oracle.RefScene(scene).render(cam, cfg, sample_count=8)
    b, _, _ = oracle.RefScene(scene, det=True).render(cam, cfg, sample_count=8)
    assert relative_rmse(a, b) < 0.05


def test_reference_config_matches_library_defaults():
    """oracle.reference_config (the CPU reference arm's config, built without
    the B200 library) equals wf_render_config_default field by field."""
    import ctypes
    import wfpt
    from wfpt import abi
    a = oracle.reference_config(1920, 1080)
    b = wfpt.render_config(1920, 1080)
    assert ctypes.string_at(ctypes.addressof(a), ctypes.sizeof(a)) == \
        ctypes.string_at(ctypes.addressof(b), ctypes.sizeof(b))
    a = oracle.reference_config(64, 32, max_depth=5, caustics=1, photon_grid_min=(0, 0, 0))
    b = wfpt.render_config(64, 32, max_depth=5, caustics=1, photon_grid_min=(0, 0, 0))
    assert bytes(a) == bytes(b)
    assert ctypes.sizeof(a) == ctypes.sizeof(abi.RenderConfig)
