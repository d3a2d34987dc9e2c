"""Batches: many physical-mode jobs over several scenes in one CUDA graph per
frame (myrt_batch_*), and the autotuner that picks their launch shape.

Per-job results must equal the unbatched renders bit for bit, with any wave
size: each path's random numbers depend only on (pixel, sample, seed), and
every pixel accumulates its samples in sample order.
"""
import json

import numpy as np
import pytest

from myrt_b200 import autotune
from myrt_b200.camera import look_at
from myrt_b200.scenes import area_light, guiding_box, heightfield, icosphere_field_lit, pbr_material


class _FakeBatch:
    """Stands in for myrt_b200.Batch: frame time depends on the tuning."""

    def __init__(self):
        self._jobs = [dict(scene=0, width=8, height=8, spp=1, inverse_view=np.eye(4), inverse_projection=np.eye(4))]
        self.tuning = None
        self.renders = 0
        self.resets = 0

    def set_tuning(self, w, b):
        self.tuning = (w, b)

    def render(self):
        self.renders += 1

    def reset(self):
        self.resets += 1


def test_autotune_picks_fastest_and_caches(tmp_path, monkeypatch):
    cost = {(1 << 20, 4): 3.0, (1 << 20, 8): 2.0, (4 << 20, 4): 1.5, (4 << 20, 8): 2.5}
    monkeypatch.setattr(autotune, "time_frame", lambda b, reps=2: cost[b.tuning])
    fb = _FakeBatch()
    cache = tmp_path / "tune.json"
    r = autotune.tune_batch(fb, waves=(1 << 20, 4 << 20), blocks=(4, 8), cache=str(cache), device_name="dev")
    assert (r["wave_paths"], r["blocks_per_sm"]) == (4 << 20, 4) and fb.tuning == (4 << 20, 4)
    assert len(r["results"]) == 4 and fb.resets >= 4
    data = json.loads(cache.read_text())
    assert list(data.values())[0]["wave_paths"] == 4 << 20
    fb2 = _FakeBatch()
    monkeypatch.setattr(autotune, "time_frame", lambda b, reps=2: pytest.fail("cached: no timing"))
    r2 = autotune.tune_batch(fb2, waves=(1 << 20, 4 << 20), blocks=(4, 8), cache=str(cache), device_name="dev")
    assert r2["cached"] and fb2.tuning == (4 << 20, 4) and fb2.renders == 0


def _scenes():
    import myrt_b200 as mb

    a, la = icosphere_field_lit(n_spheres=16, subdiv=2, floor_cells=4, seed=3)
    idx, pts = heightfield(24, seed=5)
    b = dict(indices=idx, vertices=pts, materials=np.array([[0, 0]], np.int32),
             material_data=pbr_material([0.7, 0.6, 0.5], ior=1.5, roughness=0.3))
    lb = np.stack([area_light((0.3, 1.2, 0.1), 0.3, [30.0, 20.0, 10.0]),
                   area_light((-0.5, 0.8, -0.4), 0.1, [5.0, 5.0, 40.0])])
    c, lc = guiding_box(slab_cells=16, wall_cells=4)
    ctxs = []
    for s, l in ((a, la), (b, lb), (c, lc)):
        ctx = mb.Context()
        ctx.upload_scene(**s)
        ctx.set_area_lights(l)
        ctxs.append(ctx)
    return ctxs


def _jobs():
    def cam(eye, tgt, vfov, w, h):
        iv, ip = look_at(eye, tgt, vfov_deg=vfov, aspect=w / h)
        return dict(inverse_view=iv, inverse_projection=ip, width=w, height=h)

    return [
        dict(scene=0, spp=5, seed=1, **cam((0, 1, -4.5), (0, -0.3, 0), 50, 64, 48)),
        dict(scene=1, spp=3, seed=7, fp64=True, **cam((0, 1.5, -2.5), (0, 0, 0), 60, 40, 40)),
        dict(scene=2, spp=8, seed=3, max_depth=12, **cam((0, 0, -0.95), (0, 0, 0.5), 90, 96, 32)),
        dict(scene=0, spp=1, seed=2, env=(0.1, 0.1, 0.1), **cam((1, 0.5, -3), (0, 0, 0), 40, 20, 20)),
        dict(scene=1, spp=2, seed=9, max_depth=4, rr_start=1, **cam((0.5, 1.0, -2), (0, 0, 0), 70, 128, 64)),
    ]


def _unbatched(ctxs, j, frames):
    ctx = ctxs[j["scene"]]
    ctx.reset_accumulation()
    for _ in range(frames):
        ctx.render_physical(j["inverse_view"], j["inverse_projection"], j["width"], j["height"], spp=j["spp"],
                            max_depth=j.get("max_depth", 8), rr_start=j.get("rr_start", 3), seed=j.get("seed", 0),
                            env=j.get("env", (0, 0, 0)), fp64=j.get("fp64", False))
    if j.get("fp64"):
        return ctx.read_accumulation_f64(j["width"], j["height"])
    return ctx.read_accumulation(j["width"], j["height"])[0]


@pytest.mark.gpu
def test_batch_equals_unbatched():
    import myrt_b200 as mb

    ctxs = _scenes()
    jobs = _jobs()
    batch = mb.Batch(ctxs, jobs)
    batch.set_tuning(wave_paths=6000, blocks_per_sm=8)  # forces packing, and a job larger than a wave
    batch.render()
    batch.render()
    info = batch.info()
    assert info["waves"] > 3 and info["graph_nodes"] > 20
    assert info["paths_per_frame"] == sum(j["width"] * j["height"] * j["spp"] for j in jobs)
    st = batch.render_stats()
    assert st["paths"] == 2 * info["paths_per_frame"] and st["extension_rays"] >= st["paths"]
    got = [batch.read(k) for k in range(len(jobs))]
    for k, j in enumerate(jobs):
        ref = _unbatched(ctxs, j, 2)
        assert np.array_equal(got[k], ref), k
        assert np.all(got[k][..., 3] == 2 * j["spp"])
    # another launch shape renders the same images
    batch.set_tuning(wave_paths=1 << 20, blocks_per_sm=4)
    batch.reset()
    batch.render()
    batch.render()
    assert batch.info()["waves"] == 1
    for k in range(len(jobs)):
        assert np.array_equal(batch.read(k), got[k]), k
    batch.close()
    for c in ctxs:
        c.close()


@pytest.mark.gpu
def test_batch_autotune_on_device(tmp_path):
    import myrt_b200 as mb

    ctxs = _scenes()
    batch = mb.Batch(ctxs, _jobs())
    r = autotune.tune_batch(batch, waves=(4096, 1 << 16), blocks=(4, 8), reps=1, cache=str(tmp_path / "t.json"))
    assert r["ms"] > 0 and len(r["results"]) == 4
    batch.render()
    assert batch.read(0)[..., 3].max() == 5
    batch.close()
    for c in ctxs:
        c.close()
