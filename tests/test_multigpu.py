"""Renders split over ranks by sample index (myrt_b200/multigpu.py).

CPU: world_size 2 and 3 over gloo, each rank rendering its slice with the
oracle and reducing with the same all-reduce the GPU path uses; a rank that
leaves before the collective makes the other rank's all-reduce fail instead
of waiting for ever. GPU (one device): myrt_begin_samples numbers the samples
of a slice exactly as the oracle does, and render_sharded over a one-rank
NCCL group returns the full render.
"""
import multiprocessing as mp
import os
import socket
import tempfile
from datetime import timedelta
from pathlib import Path

import numpy as np
import pytest

import pyoracle as po
from myrt_b200.camera import look_at
from myrt_b200.multigpu import allreduce_accumulation, sample_slice
from myrt_b200.scenes import icosphere_field_lit

W, H = 24, 16
VIEW = dict(eye=(0, 1, -4.5), target=(0, -0.3, 0))
KW = dict(env=(0.05, 0.06, 0.08), max_depth=6, rr_start=3, seed=13)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scene():
    return icosphere_field_lit(n_spheres=6, subdiv=1, floor_cells=2, seed=4)


def _camera():
    return look_at(VIEW["eye"], VIEW["target"], vfov_deg=50, aspect=W / H)


def _gloo_rank(rank: int, world: int, port: int, spp: int, out: str, leave: int):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20))
    if rank == leave:
        os._exit(0)  # leaves without taking part in the collective
    s, lights = _scene()
    iv, ip = _camera()
    first, count = sample_slice(spp, rank, world)
    acc = (po.render_physical(s, W, H, count, iv, ip, lights, sample0=first, fp64=True, **KW) if count
           else np.zeros((H, W, 4), np.float64))
    t = torch.from_numpy(acc)
    try:
        allreduce_accumulation(t)
    except Exception as e:  # noqa: BLE001 - the peer left: report, do not hang
        Path(out + f".err{rank}").write_text(type(e).__name__)
        os._exit(3)
    if rank == 0:
        np.save(out, t.numpy())
    dist.destroy_process_group()


def _run_ranks(world: int, spp: int, leave: int = -1):
    out = os.path.join(tempfile.mkdtemp(), "acc.npy")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, spp, out, leave)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    return out, [p.exitcode for p in procs]


def test_sample_slices_partition_the_samples():
    for spp in (0, 1, 5, 64, 1001):
        for world in (1, 2, 3, 8):
            got = [sample_slice(spp, r, world) for r in range(world)]
            idx = [i for first, count in got for i in range(first, first + count)]
            assert idx == list(range(spp))
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        sample_slice(4, 2, 2)


@pytest.mark.parametrize("world,spp", [(2, 5), (3, 2)])
def test_gloo_sharded_render_equals_full_render(world, spp):
    out, codes = _run_ranks(world, spp)
    assert codes == [0] * world, codes
    got = np.load(out)
    s, lights = _scene()
    iv, ip = _camera()
    ref = po.render_physical(s, W, H, spp, iv, ip, lights, fp64=True, **KW)
    assert np.array_equal(got[..., 3], ref[..., 3])
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-300)


def test_gloo_rank_that_leaves_fails_the_collective():
    out, codes = _run_ranks(2, 4, leave=1)
    assert codes[1] == 0
    assert codes[0] == 3, codes  # rank 0's all-reduce raised instead of waiting
    assert Path(out + ".err0").exists()


@pytest.mark.gpu
def test_begin_samples_numbers_a_slice(ctx):
    s, lights = _scene()
    ctx.upload_scene(**s)
    ctx.set_area_lights(lights)
    iv, ip = _camera()
    ctx.render_physical(iv, ip, W, H, spp=3, **KW)  # something to overwrite
    ctx.begin_samples(5)
    ctx.render_physical(iv, ip, W, H, spp=4, **KW)
    assert ctx.sample_count() == 9
    acc, _ = ctx.read_accumulation(W, H)
    ref = po.render_physical(s, W, H, 4, iv, ip, lights, sample0=5, **KW)
    assert np.array_equal(acc, ref)


@pytest.mark.gpu
def test_render_sharded_one_rank_nccl(ctx):
    import torch
    import torch.distributed as dist

    from myrt_b200.multigpu import render_sharded, resolve

    s, lights = _scene()
    ctx.upload_scene(**s)
    ctx.set_area_lights(lights)
    iv, ip = _camera()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60))
    try:
        acc = render_sharded(ctx, iv, ip, W, H, 6, **KW)
        torch.cuda.synchronize()
        got = acc.cpu().numpy()
        img = resolve(acc).cpu().numpy()
    finally:
        dist.destroy_process_group()
    ref = po.render_physical(s, W, H, 6, iv, ip, lights, fp64=True, **KW)
    assert np.array_equal(got[..., 3], ref[..., 3])
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-300)
    assert np.allclose(img, ref[..., :3] / ref[..., 3:4], rtol=1e-12)
