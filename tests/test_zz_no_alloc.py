"""cg_render_noalloc: rendering for callers that cannot allocate device memory.

Such a caller (a plugin handed buffers by a host application that owns the
device memory budget, code under an allocator that forbids driver
allocations mid-frame) passes its own device film; the library's queues live
in a fixed device array.  The result must equal the allocating batched entry
point's for the same view and seed, on two calls in a row (the second call
reuses the array the first one left behind).  This file is collected last so
that a failure here does not hide the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from crystalgraphics_b200 import _abi, scenes
from crystalgraphics_b200 import backend as B

pytestmark = pytest.mark.gpu
RTOL = 1e-4  # float atomic-add order, as in the other form tests

B.lib.cg_render_noalloc.restype = C.c_int
B.lib.cg_render_noalloc.argtypes = [C.c_void_p, C.POINTER(_abi.CgConf), C.POINTER(_abi.CgViewDesc),
                                    C.c_void_p, C.c_void_p, C.c_void_p]


def _view_desc(cam, w, h, spp, seed):
    arr = B.make_views([(cam.position[:], cam.direction[:], w, h, spp, seed,
                         tuple(cam.viewport[:]))])
    return arr[0]


@pytest.mark.parametrize("make,depth,spp", [(lambda: scenes.cornell(), 3, 4),
                                            (lambda: scenes.icosphere_scene(subdiv=4), 8, 8)])
def test_noalloc_matches_allocating_entry_point_on_two_calls(make, depth, spp):
    import torch
    W, H, seed = 96, 64, 4321
    conf = B.PathTraceConf(render_width=W, render_height=H, sample_count=spp, trace_depth=depth)
    B.EnvInit(conf)
    s = make()
    g = B.LoadScene(s)
    vd = _view_desc(s.camera, W, H, spp, seed)
    ref = B.batch_render(g, [(s.camera.position[:], s.camera.direction[:], W, H, spp, seed,
                              tuple(s.camera.viewport[:]))])[0]
    film = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    rgba = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    cconf = conf.to_c()
    scale = max(float(np.abs(ref).mean()), 1e-6)
    for call in range(2):
        film.fill_(float("nan"))  # every pixel must be written
        rgba.fill_(0)
        torch.cuda.synchronize()
        rc = B.lib.cg_render_noalloc(g.handle, C.byref(cconf), C.byref(vd), film.data_ptr(),
                                     rgba.data_ptr(), None)
        assert rc == 0, B.lib.cg_last_error().decode()
        torch.cuda.synchronize()
        out = film.cpu().numpy()
        assert np.all(np.isfinite(out)), call
        assert float(np.abs(out[..., :3] - ref).max()) / scale < RTOL, call
        assert int(rgba.cpu().numpy()[..., 3].min()) == 255
    g.close()
    B.EnvTerm()


def test_noalloc_rejects_a_view_beyond_its_scratch():
    import torch
    conf = B.PathTraceConf(render_width=8, render_height=8, sample_count=1, trace_depth=12)
    B.EnvInit(conf)
    s = scenes.cornell()
    g = B.LoadScene(s)
    vd = _view_desc(s.camera, 8, 8, 1 << 20, 1)
    film = torch.empty((8, 8, 4), dtype=torch.float32, device="cuda")
    cconf = conf.to_c()
    rc = B.lib.cg_render_noalloc(g.handle, C.byref(cconf), C.byref(vd), film.data_ptr(), None, None)
    assert rc == _abi.CG_E_INVALID
    assert "exceeds the no-alloc scratch" in B.lib.cg_last_error().decode()
    g.close()
    B.EnvTerm()
