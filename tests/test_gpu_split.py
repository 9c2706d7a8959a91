"""One view split across GPUs, on one GPU: sample ranges of a frame add up
to the full View() frame, the device film is the film ReadFilm returns, and
ViewSplit in a one-rank NCCL group reproduces View().

Sample keys depend on (seed, frame, pixel, sample index), and a range's film
holds each of its samples' terms divided by the full frame's spp, so the
films of ranges that partition the samples sum to the full frame up to the
order of float additions.
"""
import os
import socket

import numpy as np
import pytest

from crystalgraphics_b200 import _abi, scenes
from crystalgraphics_b200 import backend as B

from gpu_common import small_instanced

pytestmark = pytest.mark.gpu
RTOL = 1e-4  # float addition order


def _close(a, b):
    scale = max(float(np.abs(b).mean()), 1e-6)
    return float(np.abs(a - b).max()) / scale


@pytest.fixture(scope="module")
def scene_pair():
    B.EnvInit(B.PathTraceConf(render_width=64, render_height=64, sample_count=1, trace_depth=3))
    s1, s2 = scenes.cornell(), small_instanced()
    g1, g2 = B.LoadScene(s1), B.LoadScene(s2)
    yield [(s1, g1), (s2, g2)]
    g1.close()
    g2.close()
    B.EnvTerm()


@pytest.mark.parametrize("which", [0, 1])
def test_sample_ranges_add_up_to_the_full_frame(scene_pair, which):
    s, g = scene_pair[which]
    B.EnvInit(B.PathTraceConf(render_width=96, render_height=80, sample_count=6, trace_depth=4))
    cam = B.Camera.from_c(s.camera)
    B.View(g, cam)
    full = B.ReadFilm()
    assert float(np.abs(full).max()) > 0
    parts = []
    for begin, count in ((0, 2), (2, 1), (3, 3)):
        B.ViewSamples(g, cam, begin, count)
        parts.append(B.ReadFilm())
    assert _close(parts[0] + parts[1] + parts[2], full) < RTOL
    B.ViewSamples(g, cam, 0, 6)
    assert _close(B.ReadFilm(), full) < RTOL
    B.ViewSamples(g, cam, 6, 0)
    assert not B.ReadFilm().any()
    with pytest.raises(B.Error) as e:
        B.ViewSamples(g, cam, 4, 3)
    assert e.value.code == _abi.CG_E_INVALID
    B.View(g, cam)  # a share restarts the running mean
    assert B.FilmFrames() == 1


def test_device_film_and_rgba8_update(scene_pair):
    import torch
    s, g = scene_pair[0]
    B.EnvInit(B.PathTraceConf(render_width=72, render_height=40, sample_count=3, trace_depth=3))
    cam = B.Camera.from_c(s.camera)
    B.View(g, cam)
    rgba = B.ReadFilm(_abi.CG_FILM_RGBA8)
    film = B.FilmDevice()
    assert film.shape == (40, 72, 4) and film.dtype == torch.float32 and film.is_cuda
    np.testing.assert_array_equal(film[..., :3].cpu().numpy(), B.ReadFilm())
    B.UpdateRgba8()  # the same float film resolves to the same rgba8
    np.testing.assert_array_equal(B.ReadFilm(_abi.CG_FILM_RGBA8), rgba)
    film.mul_(0.0)
    torch.cuda.synchronize()
    B.UpdateRgba8()
    out = B.ReadFilm(_abi.CG_FILM_RGBA8)
    assert not out[..., :3].any() and (out[..., 3] == 255).all()


def test_view_split_in_a_one_rank_nccl_group(scene_pair):
    import torch
    import torch.distributed as dist
    s, g = scene_pair[1]
    B.EnvInit(B.PathTraceConf(render_width=80, render_height=64, sample_count=4, trace_depth=4))
    cam = B.Camera.from_c(s.camera)
    B.View(g, cam)
    full = B.ReadFilm()
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        B.ViewSplit(g, cam)
        assert _close(B.ReadFilm(), full) < RTOL
    finally:
        dist.destroy_process_group()


def test_batch_shares_render_the_films_of_the_whole_batch(scene_pair):
    """The views of a batch split over two ranks (partition_views), each share
    rendered as its own batch one after the other on this GPU, give every
    view the film the whole batch gives it."""
    _, g = scene_pair[1]
    views = [(p, d, max(8, w // 16), max(8, h // 16), spp, seed)
             for p, d, w, h, spp, seed in scenes.batch_views(24, seed=12)]
    B.EnvInit(B.PathTraceConf(render_width=64, render_height=64, sample_count=1, trace_depth=4))
    whole = B.batch_render(g, views)
    parts = B.partition_views(views, 2)
    assert sorted(parts[0] + parts[1]) == list(range(len(views))) and parts[0] and parts[1]
    for part in parts:
        films = B.batch_render(g, [views[k] for k in part])
        for k, f in zip(part, films):
            assert _close(f, whole[k]) < RTOL, k


def test_routed_requests_render_the_films_of_one_server(scene_pair):
    """A request stream routed over two ranks (RequestRouter), each rank's
    requests served by its own server (one after the other on this GPU),
    gives every request the film one server gives it."""
    gs = [g for _, g in scene_pair]
    stream = [(t, si % 2, p, d, w // 8, h // 8, spp, seed)
              for t, si, p, d, w, h, spp, seed in scenes.request_stream(12, 100.0, seed=13)]
    B.EnvInit(B.PathTraceConf(render_width=64, render_height=64, sample_count=16, trace_depth=4))

    def serve(reqs):
        with B.Server(gs, 8 << 30) as sv:
            ids = [sv.submit(si, p, d, w, h, spp, seed) for _, si, p, d, w, h, spp, seed in reqs]
            return [sv.wait(i)[0] for i in ids]

    one = serve(stream)
    router = B.RequestRouter(2)
    owner = [router.route(w, h, spp) for _, _, _, _, w, h, spp, _ in stream]
    assert set(owner) == {0, 1}
    for rank in (0, 1):
        ks = [k for k in range(len(stream)) if owner[k] == rank]
        for k, f in zip(ks, serve([stream[k] for k in ks])):
            assert _close(f, one[k]) < RTOL, k
