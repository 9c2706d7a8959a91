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
import os
import subprocess
import sys
import textwrap

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
        # per value, against its own size plus the film's mean: the sample
        # trees' terms reach a sample slot in another order here, and on the
        # depth-8 icosphere a bright pixel's 1e-6 relative reordering error is
        # above 1e-4 of the film's mean
        err = np.abs(out[..., :3] - ref) / (np.abs(ref) + scale)
        assert float(err.max()) < RTOL, call
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


def _cudart():
    """The CUDA runtime the library itself loaded (same soname), for device
    buffers that are exactly as large as asked (torch's allocator pools them)."""
    rt = C.CDLL("libcudart.so.12")
    rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    rt.cudaFree.argtypes = [C.c_void_p]
    return rt


def test_noalloc_rejects_bad_films_and_sizes_before_any_launch():
    """A film in host memory, a device film too small for the view and a view
    of more than 2^32 - 1 pixels are turned into CG_E_INVALID on the host; no
    kernel runs for them."""
    conf = B.PathTraceConf(render_width=8, render_height=8, sample_count=1, trace_depth=2)
    B.EnvInit(conf)
    s = scenes.cornell()
    g = B.LoadScene(s)
    cconf = conf.to_c()
    host = np.zeros((8, 8, 4), np.float32)
    vd = _view_desc(s.camera, 8, 8, 1, 1)
    rc = B.lib.cg_render_noalloc(g.handle, C.byref(cconf), C.byref(vd), host.ctypes.data, None,
                                 None)
    assert rc == _abi.CG_E_INVALID
    assert "film_xyzw" in B.lib.cg_last_error().decode()
    rt = _cudart()
    small = C.c_void_p()
    assert rt.cudaMalloc(C.byref(small), 4096) == 0
    try:
        big = _view_desc(s.camera, 1024, 1024, 1, 1)       # needs 16 MiB of film
        rc = B.lib.cg_render_noalloc(g.handle, C.byref(cconf), C.byref(big), small.value, None,
                                     None)
        assert rc == _abi.CG_E_INVALID
        assert "bytes from its start" in B.lib.cg_last_error().decode()
        huge = _view_desc(s.camera, 65536, 65536, 1, 1)    # 2^32 pixels
        rc = B.lib.cg_render_noalloc(g.handle, C.byref(cconf), C.byref(huge), small.value, None,
                                     None)
        assert rc == _abi.CG_E_INVALID
        assert "2^32" in B.lib.cg_last_error().decode()
    finally:
        rt.cudaFree(small)
    g.close()
    B.EnvTerm()


_CONTEXT_CHILD = textwrap.dedent("""
    import ctypes as C, os, sys
    sys.path.insert(0, sys.argv[1])
    import numpy as np
    from crystalgraphics_b200 import _abi, scenes
    from crystalgraphics_b200 import backend as B
    L = B.lib
    L.cg_render_noalloc.restype = C.c_int
    L.cg_render_noalloc.argtypes = [C.c_void_p, C.POINTER(_abi.CgConf), C.POINTER(_abi.CgViewDesc),
                                    C.c_void_p, C.c_void_p, C.c_void_p]
    rt = C.CDLL("libcudart.so.12")
    rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    W, H = 32, 24
    conf = B.PathTraceConf(render_width=W, render_height=H, sample_count=2, trace_depth=3)
    s = scenes.cornell()
    vd = B.make_views([(s.camera.position[:], s.camera.direction[:], W, H, 2, 77,
                        tuple(s.camera.viewport[:]))])[0]
    cconf = conf.to_c()

    def render(scene):
        film = C.c_void_p()
        assert rt.cudaMalloc(C.byref(film), W * H * 16) == 0
        rc = L.cg_render_noalloc(scene.handle, C.byref(cconf), C.byref(vd), film.value, None, None)
        out = np.zeros((H, W, 4), np.float32)
        if rc == 0:
            assert rt.cudaMemcpy(out.ctypes.data, film.value, W * H * 16, 2) == 0
        return rc, out

    B.EnvInit(conf)
    g = B.LoadScene(s)
    rc, before = render(g)
    assert rc == 0, L.cg_last_error().decode()
    B.EnvTerm()
    assert rt.cudaDeviceReset() == 0          # ends this process's context only
    B.EnvInit(conf)
    rc, _ = render(g)                         # the scene's buffers died with the old context
    assert rc == _abi.CG_E_INVALID, rc
    assert "another CUDA context" in L.cg_last_error().decode()
    g2 = B.LoadScene(s)                       # uploaded in the new context
    rc, after = render(g2)                    # the scratch is set up again there
    assert rc == 0, L.cg_last_error().decode()
    scale = max(float(np.abs(before).mean()), 1e-6)
    assert np.all(np.isfinite(after))
    assert float(np.abs(after - before).max()) / scale < 1e-4
    print("CONTEXT_OK", flush=True)
    os._exit(0)                               # the first scene's handles are stale: skip teardown
""")


def test_noalloc_follows_a_new_context_and_rejects_stale_scenes():
    """After a device reset (a new CUDA context on the same device) a scene
    uploaded before it is rejected, and the scratch is set up again for the new
    context, so a scene uploaded there renders the same film as before.  Runs
    in a child process: the reset ends that process's context only."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _CONTEXT_CHILD, root], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0 and "CONTEXT_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
