"""The benchmark's two arms measure the same workload (CPU).

The closest-hit batch is counter-based: any subset of ray indices regenerates
exactly the batch's own camera rays and bounce rays, so the reference arm's
samples are rays of the batch. The reference arm prints the same `config` as
the library's arm and never maps the CUDA library.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

from myrt_b200.scenes import diffuse_bounce_rays, jittered_camera_rays

ROOT = Path(__file__).resolve().parents[1]


def test_camera_rays_of_a_subset_equal_the_batch_rows():
    full = jittered_camera_rays(np.arange(4096), 32, seed=1000)
    idx = np.array([4095, 7, 1000, 7, 0])
    assert np.array_equal(jittered_camera_rays(idx, 32, seed=1000), full[idx])
    assert not np.array_equal(jittered_camera_rays(idx, 32, seed=1001), full[idx])
    d = full[:, 4:7].astype(np.float64)
    assert np.allclose((d * d).sum(1), 1.0, atol=1e-6)


def test_bounce_rays_depend_only_on_the_parent_index():
    rng = np.random.default_rng(0)
    tris9 = rng.uniform(-1, 1, (10, 9)).astype(np.float32)
    rays = jittered_camera_rays(np.arange(64), 8, seed=3)
    prim = rng.integers(0, 10, 64).astype(np.int32)
    t = rng.uniform(1, 2, 64).astype(np.float32)
    idx = np.arange(64)
    a = diffuse_bounce_rays(rays, prim, t, tris9, idx, seed=3)
    sel = np.array([5, 60, 1])
    b = diffuse_bounce_rays(rays[sel], prim[sel], t[sel], tris9, idx[sel], seed=3)
    assert np.array_equal(a[sel], b)


def test_reference_arm_prints_the_library_arms_config_without_the_cuda_library():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1")
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, env=env, cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([x for x in out.stdout.splitlines() if x.startswith("{")][-1])
    sys.path.insert(0, str(ROOT))
    import bench

    assert line["impl"] == "reference"
    assert line["config"] == bench.closest_config(655_872, 512, 64, 1)
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_oracle_render_with_a_prepared_scene_equals_a_fresh_one():
    """The render workload times the oracle's passes with the scene prepared
    (baked and its tree built) beforehand; the image is the same."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle as po
    from myrt_b200.camera import look_at
    from myrt_b200.scenes import icosphere_field

    s = icosphere_field(n_spheres=6, subdiv=1, floor_cells=2, seed=3)
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=1.5)
    a, da = po.render_reference(s, 24, 16, 3, 2, iv, ip, seed=9)
    b, db = po.render_reference(s, 24, 16, 3, 2, iv, ip, seed=9, prepared=po.prepare_reference(s))
    assert np.array_equal(a, b) and np.array_equal(da, db)
    assert a[..., 3].min() == 2
