"""Closest-hit and shadow any-hit kernels against the host-compiled reference.

Ray queries involve no elementary functions, so the CUDA kernels must agree
with the reference's traceRay/isOccluded bit for bit: t, position, normals,
material and light index (hit records), primitive and instance identity
(through the reference's probe-scene encoding), and the occlusion flag."""
import numpy as np
import pytest

import oracle
import wfpt
from wfpt import abi, scenes
from helpers import acceleration_cases, acceleration_rays, camera_rays, hit_diff

pytestmark = pytest.mark.gpu

CASES = acceleration_cases()


def compare(scene, rays):
    dev = wfpt.DeviceScene(scene)
    got = dev.trace_closest(rays)
    ref = oracle.RefScene(scene, det=True)
    want = ref.trace(rays)
    bad = hit_diff(got, want)
    assert len(bad) == 0, f"{len(bad)} hit records differ, first {bad[:5]}: {got[bad[:2]]} vs {want[bad[:2]]}"
    probe = oracle.RefScene(scene, det=True, probe=True).trace(rays)
    assert np.array_equal(got["kind"], probe["kind"])
    hit = got["kind"] != abi.HIT_NONE
    assert np.array_equal(got["primitive"][hit], probe["primitive"][hit])
    mesh = got["kind"] == abi.HIT_MESH
    assert np.array_equal(got["instance"][mesh], probe["instance"][mesh])
    # isOccluded just before / after the closest hit (scene_acceleration_tests.cu:128-135).
    limit = np.where(hit, want["t"], np.float32(1000.0)).astype(np.float32)
    for delta in (-0.02, 0.02):
        md = (limit + np.float32(delta)).astype(np.float32)
        occ = dev.trace_any(rays, md)
        assert np.array_equal(occ, ref.occluded(rays, md))
    dev.close()
    return got


@pytest.mark.parametrize("name", list(CASES))
def test_acceleration_cases(cuda, name):
    got = compare(CASES[name], acceleration_rays())
    if name == "empty scene":
        assert (got["kind"] == abi.HIT_NONE).all()


def test_cornell_camera_and_random_rays(cuda):
    scene, cam = scenes.cornell_box(128, 128)
    compare(scene, camera_rays(cam, 128, 128))
    rays = acceleration_rays(seed=7, count=20000)
    rays["origin"] = rays["origin"] * np.float32(0.6) + np.float32([0, 1, 0])
    compare(scene, rays)


def test_sphere_field_rays(cuda):
    scene, cam = scenes.sphere_field(160, 90, frequency=24)
    got = compare(scene, camera_rays(cam, 160, 90))
    kinds = set(np.unique(got["kind"]).tolist())
    assert {abi.HIT_SPHERE, abi.HIT_MESH} <= kinds


def test_large_mesh_rays(cuda):
    scene, cam = scenes.large_mesh(128, 72, terrain_quads=96, instance_count=24, instance_frequency=10,
                                   glass_spheres=4, env_size=(128, 64))
    got = compare(scene, camera_rays(cam, 128, 72))
    assert (got["kind"] == abi.HIT_MESH).mean() > 0.5
