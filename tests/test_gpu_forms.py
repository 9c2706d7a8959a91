"""The batched and served forms, the autotuner and the C++ layer on the GPU.

Per-sample streams are keyed by (seed, frame, pixel, sample), so a view
rendered alone, in a batch, or as a served request in a mix produces the same
samples; results agree up to the order of float atomic additions.
"""
import os
import subprocess
import time

import numpy as np
import pytest

from crystalgraphics_b200 import _abi, film_io, gltf, scenes
from crystalgraphics_b200 import backend as B

from gpu_common import small_instanced

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RTOL = 1e-4  # float atomic-add order


@pytest.fixture(scope="module")
def cornell():
    B.EnvInit(B.PathTraceConf(render_width=64, render_height=64, sample_count=1, trace_depth=3))
    s = scenes.cornell()
    g = B.LoadScene(s)
    yield s, g
    g.close()
    B.EnvTerm()


def _views(s):
    cam = s.camera
    sizes = [(33, 17, 1), (64, 64, 4), (100, 40, 2), (16, 16, 8), (128, 96, 3)]
    return [(cam.position[:], cam.direction[:], w, h, spp, 77 + k, (0.5 * w / h, 0.5))
            for k, (w, h, spp) in enumerate(sizes)]


def _close(a, b):
    scale = max(float(np.abs(b).mean()), 1e-6)
    return float(np.abs(a - b).max()) / scale


def test_batch_matches_single_views(cornell):
    s, g = cornell
    views = _views(s)
    films = B.batch_render(g, views)
    for (pos, d, w, h, spp, seed, vp), film in zip(views, films):
        B.EnvInit(B.PathTraceConf(render_width=w, render_height=h, sample_count=spp, trace_depth=3))
        B.SetSeed(seed)
        B.View(g, B.Camera(tuple(pos), tuple(d), vp))
        single = B.ReadFilm()
        assert film.shape == single.shape
        assert _close(film, single) < RTOL, (w, h, spp)
    B.EnvInit(B.PathTraceConf(render_width=64, render_height=64, sample_count=1, trace_depth=3))


def test_film_read_formats(cornell):
    """XYZ, linear sRGB (the xyz_to_srgb matrix, each product and sum rounded
    to float32 in the same order) and rgba8 readbacks of one film, into
    pageable and pinned host buffers."""
    import torch

    s, g = cornell
    B.EnvInit(B.PathTraceConf(render_width=61, render_height=37, sample_count=2, trace_depth=3))
    B.View(g, B.Camera.from_c(s.camera))
    xyz = B.ReadFilm(_abi.CG_FILM_XYZ32F)
    rgb = B.ReadFilm(_abi.CG_FILM_RGB32F)
    pinned = torch.empty((37, 61, 3), dtype=torch.float32, pin_memory=True).numpy()
    B.ReadFilm(_abi.CG_FILM_XYZ32F, out=pinned)
    assert np.array_equal(pinned, xyz)
    assert float(np.abs(xyz).max()) > 0
    f = np.float32
    X, Y, Z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    m = [(2.36461385, -0.89654057, -0.46807328), (-0.51516621, 1.4264081, 0.0887581),
         (0.0052037, -0.01440816, 1.00920446)]
    for c, (a, b, d) in enumerate(m):
        want = (f(a) * X + f(b) * Y) + f(d) * Z
        assert np.array_equal(rgb[..., c], want), c
    rgba = B.ReadFilm(_abi.CG_FILM_RGBA8)
    assert rgba.shape == (37, 61, 4) and int(rgba[..., 3].min()) == 255
    B.EnvInit(B.PathTraceConf(render_width=64, render_height=64, sample_count=1, trace_depth=3))


def test_batch_graph_replay_is_stable(cornell):
    s, g = cornell
    B.SetTuning(use_graph=1)
    views = _views(s)
    a = B.batch_render(g, views)
    st1 = B.LastStats()
    b = B.batch_render(g, views)   # replays the captured graph
    st2 = B.LastStats()
    assert st1.samples == st2.samples == sum(w * h * spp for _, _, w, h, spp, _, _ in views)
    for x, y in zip(a, b):
        assert _close(x, y) < RTOL
    films8 = B.batch_render(g, views, rgba=True)[1]
    assert films8[1].shape == (64, 64, 4) and films8[1][..., 3].min() == 255


def test_batch_uneven_views_in_many_chunks(cornell):
    """A queue small enough that a batch needs many chunks gives the same
    films as one large chunk."""
    s, g = cornell
    views = _views(s)
    ref = B.batch_render(g, views)
    B.SetTuning(queue_capacity=8192)
    small = B.batch_render(g, views)
    assert B.LastStats().chunks > 3
    B.SetTuning(queue_capacity=64 << 20)
    for x, y in zip(ref, small):
        assert _close(x, y) < RTOL


@pytest.mark.parametrize("use_graph", [0, 1])
def test_chunk_pipelines_render_the_same_films(cornell, use_graph):
    """Chunks spread over two or three streams with their own ray queues give
    the same films (and ray counts) as one pipeline, in View() and in a
    captured batch."""
    s, g = cornell
    views = _views(s)
    conf = B.PathTraceConf(render_width=96, render_height=80, sample_count=4, trace_depth=4)
    out = {}
    for pl in (1, 2, 3):
        B.EnvInit(conf)
        B.SetTuning(queue_capacity=8192, pipelines=pl, use_graph=use_graph)
        B.View(g, B.Camera.from_c(s.camera))
        st = B.LastStats()
        assert st.chunks > 3
        out[pl] = (B.ReadFilm(), st.extend_rays, st.shadow_rays, B.batch_render(g, views))
    a = out[1]
    for pl in (2, 3):
        b = out[pl]
        assert _close(b[0], a[0]) < RTOL
        assert (a[1], a[2]) == (b[1], b[2])
        for x, y in zip(a[3], b[3]):
            assert _close(y, x) < RTOL
    B.EnvInit(B.PathTraceConf(render_width=64, render_height=64, sample_count=1, trace_depth=3))


def test_deferred_light_pdf_matches_inline(cornell):
    """With the level-wide shading order, the children of a light-sampling
    level leave the light-pdf term of their denominators to a separate pass
    (k_light_pdf); with the per-block order the shading kernel adds it itself.
    Both walk the light BVH with the same explicitly rounded arithmetic, so a
    512x512, 4 spp frame (one chunk, and several chunks with a 2^20-ray queue)
    has the same keyed samples either way."""
    s, g = cornell
    conf = B.PathTraceConf(render_width=512, render_height=512, sample_count=4, trace_depth=3)
    out = {}
    for sort, queue in (("global", 0), ("block", 1 << 20), ("global", 1 << 20)):
        B.EnvInit(conf)
        B.SetTuning(queue_capacity=queue, shade_sort=sort)
        B.View(g, B.Camera.from_c(s.camera))
        st = B.LastStats()
        out[(sort, queue)] = (B.ReadFilm(), st.chunks, st.extend_rays, st.shadow_rays)
    ref = out[("global", 0)]
    assert ref[1] == 1 and float(np.abs(ref[0]).mean()) > 0.0
    for key in (("block", 1 << 20), ("global", 1 << 20)):
        o = out[key]
        assert o[1] > 1, key
        assert (o[2], o[3]) == (ref[2], ref[3]), key
        assert _close(o[0], ref[0]) < RTOL, key
    B.EnvInit(B.PathTraceConf(render_width=64, render_height=64, sample_count=1, trace_depth=3))


def test_view_graph_replay_matches_direct_launches(cornell):
    """View() replays its captured launch sequence; accumulated frames, a
    camera change and a switch to another scene (a new capture) give the films
    of direct launches."""
    s, g = cornell
    s2 = small_instanced()
    g2 = B.LoadScene(s2)
    conf = B.PathTraceConf(render_width=80, render_height=64, sample_count=2, trace_depth=4)
    cam = B.Camera.from_c(s.camera)
    moved = B.Camera(tuple(x + 0.01 for x in s.camera.position[:]), tuple(s.camera.direction[:]),
                     (0.5 * 80 / 64, 0.5))
    films = {}
    for use_graph in (0, 1):
        B.EnvInit(conf)
        B.SetTuning(use_graph=use_graph)
        out = []
        for scene, c in ((g, cam), (g, cam), (g, cam), (g, moved), (g2, B.Camera.from_c(s2.camera)),
                         (g, cam)):
            B.View(scene, c)
            out.append((B.ReadFilm(), B.FilmFrames(), B.LastStats().kernel_launches))
        films[use_graph] = out
    for (a, fa, la), (b, fb, lb) in zip(films[0], films[1]):
        assert fa == fb and la == lb
        assert _close(b, a) < RTOL
    g2.close()
    B.EnvInit(B.PathTraceConf(render_width=64, render_height=64, sample_count=1, trace_depth=3))


def test_server_results_same_alone_and_in_the_mix(cornell):
    s, g = cornell
    s2 = small_instanced()
    g2 = B.LoadScene(s2)
    reqs = [(0, 48, 40, 4, 5), (1, 64, 48, 2, 6), (0, 32, 32, 8, 7), (1, 40, 40, 1, 8),
            (0, 80, 60, 2, 9)]
    cams = [s.camera, s2.camera]

    def submit(sv, r):
        si, w, h, spp, seed = r
        c = cams[si]
        return sv.submit(si, c.position[:], c.direction[:], w, h, spp, seed)

    alone = []
    with B.Server([g, g2], 1 << 30) as sv:
        for r in reqs:
            film, res = sv.wait(submit(sv, r))
            assert res.status == 0
            alone.append(film)
    with B.Server([g, g2], 1 << 30) as sv:
        ids = [submit(sv, r) for r in reqs]
        mixed = [sv.wait(i)[0] for i in ids]
        st = sv.stats()
        assert st.completed == len(reqs) and st.samples == sum(w * h * spp for _, w, h, spp, _ in reqs)
    for a, b in zip(alone, mixed):
        assert _close(b, a) < RTOL
    # and a served request equals the same view rendered by the batched form
    si, w, h, spp, seed = reqs[0]
    ref = B.batch_render(g, [(s.camera.position[:], s.camera.direction[:], w, h, spp, seed)])[0]
    assert _close(mixed[0], ref) < RTOL


def test_server_in_hero_mode_matches_the_batched_form(cornell):
    """A server created while hero-wavelength sampling is on keeps that mode:
    its requests equal the same views rendered by the batched form in hero
    mode, alone and in a mix, and differ from reference-mode frames."""
    s, g = cornell
    c = s.camera
    reqs = [(48, 40, 4, 15), (32, 32, 8, 16), (80, 60, 2, 17)]
    views = [(c.position[:], c.direction[:], w, h, spp, seed) for w, h, spp, seed in reqs]
    B.SetSpectral(_abi.CG_SPECTRAL_HERO)
    try:
        ref = B.batch_render(g, views)
        with B.Server([g], 1 << 30) as sv:
            ids = [sv.submit(0, c.position[:], c.direction[:], w, h, spp, seed)
                   for w, h, spp, seed in reqs]
            served = [sv.wait(i)[0] for i in ids]
    finally:
        B.SetSpectral(_abi.CG_SPECTRAL_REFERENCE)
    plain = B.batch_render(g, views)
    for a, b, p in zip(served, ref, plain):
        assert _close(a, b) < RTOL
        assert _close(p, b) > 10 * RTOL


def test_server_admission_under_budget(cornell):
    s, g = cornell
    c = s.camera
    with B.Server([g], 1 << 30) as probe:
        rid = probe.submit(0, c.position[:], c.direction[:], 64, 64, 2, 1)
        probe.wait(rid)
        one = probe.stats().peak_bytes
    assert one > 0
    budget = int(one * 1.5)  # room for one request at a time
    with B.Server([g], budget) as sv:
        ids = [sv.submit(0, c.position[:], c.direction[:], 64, 64, 2, k) for k in range(6)]
        for i in ids:
            sv.wait(i)
        st = sv.stats()
        assert st.completed == 6 and st.peak_bytes <= budget
    with B.Server([g], one // 2) as tiny:  # can never fit
        rid = tiny.submit(0, c.position[:], c.direction[:], 64, 64, 2, 1)
        with pytest.raises(B.Error) as e:
            tiny.wait(rid)
        assert e.value.code == _abi.CG_E_OOM
        assert tiny.stats().rejected == 1


def test_server_cancel_and_timeout(cornell):
    s, g = cornell
    c = s.camera
    with B.Server([g], 8 << 30) as sv:
        big = [sv.submit(0, c.position[:], c.direction[:], 512, 512, 16, k) for k in range(4)]
        last = sv.submit(0, c.position[:], c.direction[:], 512, 512, 16, 99)
        sv.cancel(last)
        with pytest.raises(B.Error) as e:
            sv.wait(last)
        assert e.value.code in (_abi.CG_E_CANCELLED,)
        try:
            sv.wait(big[-1], timeout_ms=0)
            finished = True
        except B.Error as err:
            assert err.code == _abi.CG_E_TIMEOUT
            finished = False
        for i in big[:-1]:
            sv.wait(i)
        if not finished:
            sv.wait(big[-1])
        assert sv.stats().cancelled == 1


@pytest.mark.parametrize("variant", [dict(bvh_width=2, persistent=False),
                                     dict(bvh_width=2, persistent=True),
                                     dict(bvh_width=4, persistent=True),
                                     dict(bvh_width=4, persistent=False),
                                     dict(bvh_width=4, persistent=False, shade_sort=False),
                                     dict(bvh_width=4, persistent=True, shade_sort="block"),
                                     dict(bvh_width=4, persistent=False, box_bits=8),
                                     dict(bvh_width=4, persistent="postponed"),
                                     dict(bvh_width=4, persistent=True, traversal_threads=768,
                                          pipelines=3),
                                     dict(bvh_width=4, persistent="postponed", box_bits=8)])
def test_traversal_variants_render_the_same_samples(variant):
    """Binary or four-wide trees, one ray per thread or persistent warps, rays
    grouped by material before shading or not: the closest hits and the keyed
    samples are the same, so the frames are (up to float atomic order)."""
    s = scenes.icosphere_scene(subdiv=4)
    B.EnvInit(B.PathTraceConf(render_width=96, render_height=54, sample_count=4, trace_depth=8))
    g = B.LoadScene(s)
    cam = B.Camera.from_c(s.camera)
    B.SetTuning(bvh_width=4, persistent=False, shade_sort=True, box_bits=32)
    B.View(g, cam)
    ref = B.ReadFilm()
    B.EnvInit(B.PathTraceConf(render_width=96, render_height=54, sample_count=4, trace_depth=8))
    B.SetTuning(**variant)
    B.View(g, cam)
    out = B.ReadFilm()
    st = B.LastStats()
    assert _close(out, ref) < RTOL
    assert st.extend_rays > 0 and st.shadow_rays > 0
    g.close()


def test_autotune_returns_a_valid_tuning(cornell):
    s, g = cornell
    t = B.autotune(g, (s.camera.position[:], s.camera.direction[:], 96, 96, 4, 1))
    assert t.queue_capacity >= 4096 and t.extend_block % 32 == 0 and t.shade_block % 32 == 0
    assert t.bvh_width in (2, 4) and t.box_bits in (8, 32) and t.shade_sort in (1, 2, 3)
    assert 0 < t.traversal_threads <= 1024 and t.traversal_threads % t.extend_block == 0
    # a tuning found on probe views renders the batch like the default tuning
    views = _views(s)
    ref = B.batch_render(g, views)
    t2 = B.autotune_views(g, views[::2])
    assert B.GetTuning().bvh_width == t2.bvh_width
    for x, y in zip(B.batch_render(g, views), ref):
        assert _close(x, y) < RTOL
    B.SetTuning(queue_capacity=64 << 20, extend_block=128, shade_block=128, use_graph=1,
                bvh_width=4, persistent=True, shade_sort=True, box_bits=32, pipelines=2,
                traversal_threads=1024)


def test_tuning_rejects_out_of_range_values(cornell):
    before = B.GetTuning()
    for bad in (dict(extend_block=512), dict(extend_block=48), dict(shade_block=2048),
                dict(traversal_threads=1056), dict(traversal_threads=100),
                dict(queue_capacity=1024), dict(pipelines=5), dict(bvh_width=3),
                dict(box_bits=16)):
        with pytest.raises(B.Error) as e:
            B.SetTuning(**bad)
        assert e.value.code == _abi.CG_E_INVALID, bad
    after = B.GetTuning()
    assert (after.extend_block, after.queue_capacity, after.pipelines) == \
        (before.extend_block, before.queue_capacity, before.pipelines)


def test_gltf_scene_renders_like_the_in_memory_scene(tmp_path, cornell):
    s, g = cornell
    path = gltf.write(s, str(tmp_path / "c.gltf"))
    conf = B.PathTraceConf(render_width=64, render_height=64, sample_count=4, trace_depth=3)
    B.EnvInit(conf)
    cam = B.Camera.from_c(s.camera)
    B.View(g, cam)
    a = B.ReadFilm()
    gl = B.LoadScene(path)
    B.View(gl, cam)
    b = B.ReadFilm()
    assert _close(b, a) < RTOL
    # the C++23 layer (LoadScene(path) + View + ReadFilm) end to end
    exe = os.path.join(ROOT, "crystalgraphics_b200", "cg_view")
    out = tmp_path / "c.ppm"
    args = [exe, path, str(out), "64", "64", "4", "3", "1"] + \
        [str(x) for x in list(cam.position) + list(cam.direction) + list(cam.viewport)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    img = film_io.load_ppm(out)
    # the same frame as a PFM of the linear RGB32F film
    args[2] = str(tmp_path / "c.pfm")
    r = subprocess.run(args, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lin = film_io.load_pfm(tmp_path / "c.pfm")
    B.EnvInit(conf)
    B.View(g, cam)
    ref = B.ReadFilm(_abi.CG_FILM_RGBA8)[..., :3]
    assert np.abs(img.astype(int) - ref.astype(int)).max() <= 1
    ref_lin = B.ReadFilm(_abi.CG_FILM_RGB32F)
    assert lin.shape == ref_lin.shape == (64, 64, 3)
    np.testing.assert_allclose(lin, ref_lin, rtol=1e-4, atol=1e-6 * float(np.abs(ref_lin).mean()))
