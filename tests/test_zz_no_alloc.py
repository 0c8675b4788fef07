"""luz_gpu_render_device_noalloc: rendering without device allocation.

Some hosts cannot call cudaMalloc while they render: an engine whose device
memory belongs to its own allocator, or a per-frame loop that cannot afford the
device-wide synchronisation cudaMalloc/cudaFree imply. This entry point keeps
its path state and film in a fixed file-scope device array instead. The tests
call it through the C ABI twice in a row and compare both films with the
allocating entry point (luz_gpu_render_device) on the same scene, once on an
image that fits one static wave and once on one that takes several waves
(pixel chunks of the 131,072-path arena); they also check that an image larger
than the static film is refused. The file runs last so that a
stop-at-first-failure run has executed every other test already.
"""
import ctypes as C

import numpy as np
import pytest

from cases import CASES
from luz_b200 import desc as D
from luz_b200 import native

pytestmark = pytest.mark.gpu


def _render(fn, scene, p, out, stream):
    st = D.RenderStats()
    rc = fn(scene.h, C.byref(p), C.c_void_p(out.data_ptr()), C.c_void_p(stream), C.byref(st))
    if rc != 0:
        buf = C.create_string_buffer(512)
        native.lib().luz_gpu_last_error(buf, 512)
        raise native.LuzError(rc, buf.value.decode())
    return st


def test_noalloc_matches_allocating_render_twice():
    import torch
    lib = native.lib()
    w = CASES["instancing"]()
    g = native.GpuScene(w.scene.build())
    try:
        p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
        n = w.width * w.height * 3
        stream = torch.cuda.current_stream().cuda_stream
        ref = torch.zeros(n, dtype=torch.float32, device="cuda")
        _render(lib.luz_gpu_render_device, g, p, ref, stream)
        for _ in range(2):
            out = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
            st = _render(lib.luz_gpu_render_device_noalloc, g, p, out, stream)
            torch.cuda.synchronize()
            a, b = out.cpu().numpy(), ref.cpu().numpy()
            assert np.allclose(a, b, rtol=1e-6, atol=1e-7)
            assert st.extension_rays >= w.width * w.height * w.spp and st.kernel_launches > 0
    finally:
        g.close()


def test_noalloc_multi_wave_equals_allocating_render():
    """512x288 pixels x 4 samples = 589,824 paths: five waves of the static arena
    against one wave of the allocating render. Each wave holds all four samples of
    its pixels in both, so every pixel's FP64 sum is the same sequence: equal bit
    for bit, on two calls in a row."""
    import torch
    lib = native.lib()
    w = CASES["instancing"]()
    g = native.GpuScene(w.scene.build())
    try:
        p = native.params(512, 288, 4, w.max_bounces, w.seed)
        n = 512 * 288 * 3
        stream = torch.cuda.current_stream().cuda_stream
        ref = torch.zeros(n, dtype=torch.float32, device="cuda")
        _render(lib.luz_gpu_render_device, g, p, ref, stream)
        for _ in range(2):
            out = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
            st = _render(lib.luz_gpu_render_device_noalloc, g, p, out, stream)
            torch.cuda.synchronize()
            assert st.waves == 5
            assert np.array_equal(out.cpu().numpy(), ref.cpu().numpy())
    finally:
        g.close()


def test_noalloc_rejects_image_beyond_static_film():
    import torch
    lib = native.lib()
    w = CASES["tiny"]()
    g = native.GpuScene(w.scene.build())
    try:
        p = native.params(2000, 1500, 1, 2, 1)   # 3,000,000 pixels > 2,800,000
        out = torch.zeros(3, dtype=torch.float32, device="cuda")
        with pytest.raises(native.LuzError) as e:
            _render(lib.luz_gpu_render_device_noalloc, g, p, out, torch.cuda.current_stream().cuda_stream)
        assert e.value.code == -4 and "static film" in str(e.value)
    finally:
        g.close()
