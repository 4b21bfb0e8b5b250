"""tt_render_pass_noalloc, the render pass that allocates no memory (GPU).

It serves callers that cannot let the library call cudaMalloc at render time (an
application owning all GPU memory through its own pool or budget, or code that must not
synchronise the device with an allocation).  Its path state lives in a static device array
inside the library, and it writes into device buffers the caller provides.  Here its
output is checked against the regular entry point, tt_render_pass, on the same scene and
random streams, for two calls in a row (the second call must not see the first call's
leftovers in the shared static array).  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from naivetrace_b200 import abi, scenes
from naivetrace_b200.algo import GpuContext
from naivetrace_b200.scene import make_params

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def noalloc_pass(g, spp, seed, pixel_begin, pixel_end, sample_offset=0):
    acc = torch.zeros(3 * g.npix, dtype=torch.float32, device="cuda")
    light = torch.zeros(3 * g.npix, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = g.lib.tt_render_pass_noalloc(g.h, spp, seed, pixel_begin, pixel_end, sample_offset,
                                      C.c_void_p(acc.data_ptr()), C.c_void_p(light.data_ptr()), C.c_void_p(stream))
    return st, acc.cpu().numpy().astype(np.float64), light.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("name,spp,depth", [("cornell_box", 4, 10), ("terrain_spheres_small", 8, 16),
                                            ("cornell_box_media_mix", 4, 10)])
def test_noalloc_matches_render_pass(gpu_lib, name, spp, depth):
    scene = scenes.terrain_spheres_small(64, 36) if name == "terrain_spheres_small" else getattr(scenes, name)(32, 32)
    # The allocation-free pass shades in traversal order (it has no sort buffers).
    params = make_params(max_ray_depth=depth, sort_shading=False)
    ref = GpuContext(scene, params)
    ref.render(spp, seed=7)
    acc_ref, light_ref, _, _ = ref.accumulators()
    g = GpuContext(scene, params)
    for call in range(2):
        st, acc, light = noalloc_pass(g, spp, 7, 0, g.npix)
        assert st == abi.TT_OK, abi.last_error(g.lib, g.h)
        # Same kernels and random streams; only the order of float atomic additions differs.
        np.testing.assert_allclose(acc, acc_ref, rtol=1e-5, atol=1e-6 * max(np.abs(acc_ref).max(), 1e-12))
        np.testing.assert_allclose(light, light_ref, rtol=1e-5, atol=1e-6 * max(np.abs(light_ref).max(), 1e-12))
    # The context's own accumulators are untouched by the no-allocation pass.
    acc_ctx, _, spp_ctx, splat_ctx = g.accumulators()
    assert np.all(acc_ctx == 0) and np.all(spp_ctx == 0) and splat_ctx == 0


def test_noalloc_limits(gpu_lib):
    scene = scenes.cornell_box(512, 256)
    g = GpuContext(scene, make_params(max_ray_depth=4))
    st, _, _ = noalloc_pass(g, 1, 1, 0, g.npix)  # 131072 samples > 65536
    assert st == abi.TT_ERR_CAPACITY
    assert "65536" in abi.last_error(g.lib, g.h)
    st, acc, _ = noalloc_pass(g, 1, 1, 0, 65536)
    assert st == abi.TT_OK
    assert np.abs(acc).sum() > 0


def test_noalloc_rejects_pt2(gpu_lib):
    """The null-path tracer's per-path matrices have no room in the static array."""
    g = GpuContext(scenes.cornell_box(8, 8), make_params(max_ray_depth=4, algo=abi.ALGO_PT2))
    st, _, _ = noalloc_pass(g, 1, 1, 0, g.npix)
    assert st == abi.TT_ERR_INVALID
