"""myrt_render_noalloc: the render entry point for callers that cannot call
cudaMalloc (hosts that hand all device memory to their own allocator or fixed
budgets, frame loops that must not pay cudaMalloc's implicit synchronisation).

It keeps its scratch in a static device array inside the library and writes
into images the caller owns. This test calls it through the C ABI twice in a
row (a new accumulation, then one more frame on top) and checks each result
against the allocating entry point myrt_render on the same scene, camera and
host random stream. Both run the same kernels on the same inputs, so the
images must agree bit for bit (stricter than the 1e-3 bar of the render
parity tests). A second case renders a textured scene with the environment
cube map and depth of field through a bokeh mask, on a stream the caller
owns. It uses its own contexts, so it passes alone in a fresh process as well
as after the other tests.
"""
import numpy as np
import pytest

import myrt_b200 as mb
from myrt_b200.camera import look_at
from myrt_b200.scenes import icosphere_field

pytestmark = pytest.mark.gpu


def test_render_noalloc_matches_render():
    import torch

    W, H, bounces = 128, 96, 4
    s = icosphere_field(n_spheres=24, subdiv=2, floor_cells=4, seed=4)
    iv, ip = look_at((0, 1, -4.5), (0, -0.3, 0), vfov_deg=50, aspect=W / H)
    with mb.Context(0) as ctx:
        ctx.upload_scene(**s)
        # allocating entry point: two single-frame calls
        ctx.set_seed(99)
        ctx.render(iv, ip, W, H, num_bounces=bounces, frames=1)
        ref1, disp1 = ctx.read_accumulation(W, H)
        ctx.render(iv, ip, W, H, num_bounces=bounces, frames=1)
        ref2, disp2 = ctx.read_accumulation(W, H)

        # no-allocation entry point on the same random stream, caller-owned images
        ctx.set_seed(99)
        acc = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        disp = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.render_noalloc(iv, ip, W, H, acc, disp, sample_index=0, num_bounces=bounces, frames=1)
        ctx.sync()
        got1, gdisp1 = acc.cpu().numpy(), disp.cpu().numpy()
        ctx.render_noalloc(iv, ip, W, H, acc, disp, sample_index=1, num_bounces=bounces, frames=1)
        ctx.sync()
        got2, gdisp2 = acc.cpu().numpy(), disp.cpu().numpy()

        for got, ref, gd, rd in ((got1, ref1, gdisp1, disp1), (got2, ref2, gdisp2, disp2)):
            assert np.isfinite(got).all()
            assert np.array_equal(got[..., 3], ref[..., 3])
            np.testing.assert_allclose(got, ref, rtol=0, atol=0)
            np.testing.assert_allclose(gd, rd, rtol=0, atol=0)
        assert np.all(got2[..., 3] == 2.0)

        # sizes beyond the static array are refused with a clear error
        big = torch.zeros((512, 512, 4), dtype=torch.float32, device="cuda")
        with pytest.raises(mb.MyrtError, match="65536"):
            ctx.render_noalloc(iv, ip, 512, 512, big, big, num_bounces=bounces)


def test_render_noalloc_textures_cubemap_dof_on_caller_stream():
    import torch
    from test_render_gpu import _bokeh_mask, _cubemap, _textured_heightfield

    W, H, bounces = 80, 60, 4
    scene, checker = _textured_heightfield()
    iv, ip = look_at((0, 1.2, -2.5), (0, 0, 0), vfov_deg=55, aspect=W / H)
    opts = dict(num_bounces=bounces, frames=2, dof=True, lens_size=(0.2, 0.15), focus=2.4, bokeh_slot=1)
    with mb.Context(0) as ctx:
        ctx.upload_scene(**scene)
        ctx.upload_texture(0, checker, wrap=0)
        ctx.upload_texture(1, _bokeh_mask(), wrap=0)
        ctx.upload_cubemap(_cubemap())
        ctx.set_seed(4242)
        ctx.render(iv, ip, W, H, **opts)
        ref1, disp1 = ctx.read_accumulation(W, H)
        ctx.render(iv, ip, W, H, **opts)
        ref2, disp2 = ctx.read_accumulation(W, H)

        ctx.set_seed(4242)
        stream = torch.cuda.Stream()
        acc = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        disp = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.render_noalloc(iv, ip, W, H, acc, disp, sample_index=0, stream=stream.cuda_stream, **opts)
        stream.synchronize()
        got1, gdisp1 = acc.cpu().numpy(), disp.cpu().numpy()
        ctx.render_noalloc(iv, ip, W, H, acc, disp, sample_index=2, stream=stream.cuda_stream, **opts)
        stream.synchronize()
        ctx.sync()
        got2, gdisp2 = acc.cpu().numpy(), disp.cpu().numpy()
        for got, ref, gd, rd in ((got1, ref1, gdisp1, disp1), (got2, ref2, gdisp2, disp2)):
            assert np.array_equal(got, ref)
            assert np.array_equal(gd, rd)
        assert np.all(got2[..., 3] == 4.0)
        # only the reference shading runs here, and the refusal says so
        with pytest.raises(mb.MyrtError, match="only MYRT_SHADE_REFERENCE"):
            ctx.render_noalloc(iv, ip, W, H, acc, disp, shading=1, num_bounces=bounces)
