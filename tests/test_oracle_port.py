"""Pins the oracle's own CPU restatement (oracle/pt_oracle.cpp) against the
reference's code compiled for the host: bit for bit with the C library's math
(libwfref.so) and with the deterministic math (libwfref_det.so)."""
import numpy as np
import pytest

import oracle
import wfpt
from wfpt import abi, scenes
from helpers import acceleration_cases, acceleration_rays, camera_rays, hit_diff

pytestmark = pytest.mark.skipif(not (oracle.available() and oracle.port_available()),
                                reason="oracle libraries not built")

CASES = acceleration_cases()


@pytest.mark.parametrize("name", list(CASES))
def test_port_rays_match_reference(name):
    scene = CASES[name]
    rays = acceleration_rays()
    ref = oracle.RefScene(scene)
    port = oracle.PortScene(scene)
    got, want = port.trace(rays), ref.trace(rays)
    assert len(hit_diff(got, want)) == 0
    probe = oracle.RefScene(scene, probe=True).trace(rays)
    assert np.array_equal(got["kind"], probe["kind"])
    hit = got["kind"] != abi.HIT_NONE
    assert np.array_equal(got["primitive"][hit], probe["primitive"][hit])
    limit = np.where(hit, want["t"], np.float32(1000)).astype(np.float32)
    for delta in (-0.02, 0.02):
        md = (limit + np.float32(delta)).astype(np.float32)
        assert np.array_equal(port.occluded(rays, md), ref.occluded(rays, md))


def small_large_mesh():
    return scenes.large_mesh(64, 36, terrain_quads=48, instance_count=8, instance_frequency=6, glass_spheres=3,
                             env_size=(128, 64))


RENDERS = {
    "cornell": (lambda: scenes.cornell_box(48, 48), dict(max_depth=8, rr_start_depth=3), 3),
    "sphere_field": (lambda: scenes.sphere_field(64, 36, frequency=8), dict(max_depth=16), 2),
    "large_mesh": (small_large_mesh, dict(max_depth=12), 2),
}


@pytest.mark.parametrize("det", [False, True])
@pytest.mark.parametrize("name", list(RENDERS))
def test_port_render_matches_reference(name, det):
    make, fields, spp = RENDERS[name]
    scene, cam = make()
    w = int(round(float(cam["aspect_ratio"]) * 36)) if name != "cornell" else 48
    h = 36 if name != "cornell" else 48
    cfg = wfpt.render_config(w, h, **fields)
    ref_fb, _, ref_counts = oracle.RefScene(scene, det=det).render(cam, cfg, sample_start=5, sample_count=spp)
    fb, counts = oracle.PortScene(scene, det=det).render(cam, cfg, sample_start=5, sample_count=spp)
    assert np.array_equal(fb.view(np.uint32), ref_fb.view(np.uint32))
    assert np.array_equal(counts, ref_counts)


def test_port_photons_and_caustics_match_reference():
    scene, cam = scenes.cornell_box(40, 40)
    glass = scene.add_material(wfpt.material(abi.MAT_DIELECTRIC, (1, 1, 1), ior=1.5))
    sp = np.zeros(1, abi.SPHERE_DTYPE)
    sp[0] = ((0.0, 0.4, 1.2), 0.6, glass, abi.ACCEL_BVH)
    scene.spheres = sp
    cfg = wfpt.render_config(40, 40, max_depth=8, rr_start_depth=3, caustics=1, photon_count=30000)
    ref = oracle.RefScene(scene)
    port = oracle.PortScene(scene)
    rec, _, stored = ref.photons(cfg)
    prec, pstored = port.photons(cfg)
    assert stored == pstored and stored > 100
    assert np.array_equal(prec.view(np.uint32), rec.view(np.uint32))
    a, _, _ = ref.render(cam, cfg, sample_count=2)
    b, _ = port.render(cam, cfg, sample_count=2)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
