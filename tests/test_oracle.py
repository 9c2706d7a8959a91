"""The oracle (CPU restatement of the reference) checked against the
reference's own alias_table.h fixtures and against independent Python
restatements of the reference's small formulas."""
import math
import os

import numpy as np
import pytest

import oracle as O
from crystalgraphics_b200 import _abi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_alias_matches_reference_golden():
    g = np.load(os.path.join(ROOT, "tests", "golden", "alias_tables.npz"))
    for name in sorted({k.split("__")[0] for k in g.files}):
        out = O.alias_build(g[f"{name}__w"])
        np.testing.assert_array_equal(out["alias"], g[f"{name}__alias"], err_msg=name)
        assert out["prob"].tobytes() == g[f"{name}__prob"].tobytes(), name


@pytest.mark.skipif(not O.ref_alias_available(), reason="reference tree not built here")
def test_oracle_alias_matches_reference_live():
    rng = np.random.default_rng(7)
    for n in (1, 2, 3, 17, 1000):
        w = rng.exponential(size=n)
        a = O.alias_build(w)
        r = O.ref_alias_build(w)
        assert a.tobytes() == r.tobytes()


def pcg_hash_stream(seed, n):
    """math/rng.wesl:1-22 in Python integers."""
    M = 0xFFFFFFFF

    def step(s):
        s = (s * 747796405 + 2891336453) & M
        word = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & M
        return ((word >> 22) ^ word) & M

    s = step(seed & M)
    out = []
    for _ in range(n):
        s = step(s)
        out.append(np.float32(np.float32(s) / np.float32(4294967296.0)))
    return np.array(out, np.float32), s


def test_rng_matches_python_restatement():
    import ctypes as C
    for seed in (0, 1, 123456, 0xFFFFFFFF):
        out = np.zeros(64, np.float32)
        last = O.lib().oracle_rng_sequence(seed, 64, out.ctypes.data)
        ref, s = pcg_hash_stream(seed, 64)
        np.testing.assert_array_equal(out, ref)
        assert last == s
        assert np.all(out >= 0) and np.all(out <= 1.0)


def test_wavelength_sampling_is_monotone_and_in_range():
    us = np.linspace(0, 1, 257, dtype=np.float32)
    lam = []
    for u in us:
        p = np.float32(0)
        import ctypes as C
        pc = C.c_float()
        w = O.lib().oracle_sample_wavelength(float(u), C.byref(pc))
        assert 380.0 <= w <= 720.0
        assert pc.value >= 1e-6
        lam.append(w)
    assert np.all(np.diff(lam) >= 0)


def test_xyz_match_peaks_like_cie():
    xyz = np.zeros(3, np.float32)
    best = {}
    for w in range(380, 721, 2):
        O.lib().oracle_xyz_match(float(w), xyz.ctypes.data)
        for k in range(3):
            if xyz[k] > best.get(k, (0, -1))[1]:
                best[k] = (w, float(xyz[k]))
    assert 590 <= best[0][0] <= 610   # xbar peak
    assert 550 <= best[1][0] <= 570   # ybar peak
    assert 435 <= best[2][0] <= 460   # zbar peak


def test_smits_quirk_gives_zero_in_deep_red():
    # wavelengths in [686, 720) index BINS[10]: NaN, dropped by clamp/max
    rgb = np.array([0.5, 0.5, 0.5], np.float32)
    for w in (686.5, 700.0, 719.9):
        assert O.lib().oracle_rgb_to_reflectance(rgb.ctypes.data, w) == 0.0
        assert O.lib().oracle_rgb_to_radiance(rgb.ctypes.data, w) == 0.0
    assert O.lib().oracle_rgb_to_reflectance(rgb.ctypes.data, 550.0) > 0.4


def test_emissive_buffer_weights_normalised():
    s = scenes.icosphere_scene(subdiv=2)
    os_ = O.OracleScene(s)
    prims, alias, total = os_.emissive()
    assert len(prims) == 64
    assert abs(float(prims["weight"].sum(dtype=np.float64)) - 1.0) < 1e-5
    # alias table is the reference construction on those weights
    if O.ref_alias_available():
        ref = O.ref_alias_build(prims["weight"].astype(np.float64))
        assert ref.tobytes() == alias.tobytes()


def test_oracle_closest_hit_on_axis_aligned_box():
    s = scenes.cornell()
    os_ = O.OracleScene(s)
    # a ray from the camera straight at the back wall (y = 1) through x=0.9, z=1.9
    rays = np.zeros((1, 8), np.float32)
    rays[0, :3] = (0.9, -3.0, 1.9)
    rays[0, 4:7] = (0.0, 1.0, 0.0)
    hits, t2 = os_.trace_closest(rays)
    assert hits["instance"][0] == 0  # the white walls
    assert abs(hits["t"][0] - 4.0) < 1e-5


def test_oracle_render_reference_and_keyed_agree_statistically():
    """The keyed streams change which random numbers a sample uses, not the
    estimator: both RNG orders converge to the same image (8x8-block means of
    independent frames within 3 sigma, primary-ray tie pixels left out)."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_common import pooled_masked, primary_tie_mask
    W = H = 32
    s = scenes.cornell(W, H)
    o = O.OracleScene(s)
    frames, spp = 12, 64
    conf = _abi.make_conf(W, H, spp, 2)
    keep = ~primary_tie_mask(o, s.camera, W, H)

    def run(mode, seed):
        seeds = np.zeros((H, W), np.uint32)
        out = []
        for k in range(frames):
            f, seeds, _ = o.render(conf, s.camera, film=np.zeros((H, W, 3), np.float32), seeds=seeds,
                                   iter_count=k, rng=mode, seed=seed, prune=True)
            out.append(pooled_masked(f * (k + 1), keep, 8))
        return np.stack(out)

    a, b = run(O.RNG_REFERENCE, 0), run(O.RNG_KEYED, 99)
    se = np.sqrt(a.var(0, ddof=1) / frames + b.var(0, ddof=1) / frames) + 1e-12
    z = np.abs(a.mean(0) - b.mean(0)) / se
    assert (z > 3.5).sum() <= 1, z.max()


def test_oracle_progressive_running_mean():
    s = scenes.cornell(32, 32)
    os_ = O.OracleScene(s)
    conf = _abi.make_conf(32, 32, 1, 2)
    film = np.zeros((32, 32, 3), np.float32)
    seeds = np.zeros((32, 32), np.uint32)
    f0, s0, _ = os_.render(conf, s.camera, film=film.copy(), seeds=seeds.copy(), iter_count=0,
                           rng=O.RNG_REFERENCE)
    f1, s1, _ = os_.render(conf, s.camera, film=f0.copy(), seeds=s0.copy(), iter_count=1,
                           rng=O.RNG_REFERENCE)
    assert not np.array_equal(s0, s1)
    # frame 1 holds the mean of two frames: it is between its parts on average
    assert abs(float(f1.mean()) - float(f0.mean())) < 0.5 * float(f0.mean())


def test_hero_wavelengths_cover_the_range_uniformly():
    """Four wavelengths 100 nm apart, wrapped into [380, 780]: each is uniform
    on the range when the hero is."""
    import ctypes as C
    us = np.linspace(0.0, 1.0, 4001, dtype=np.float32)
    w = np.array([[380.0 + ((400.0 * u + 100.0 * j) % 400.0) for j in range(4)] for u in us])
    assert w.min() >= 380.0 and w.max() <= 780.0
    hist, _ = np.histogram(w[:, 1:].ravel(), bins=8, range=(380, 780))
    assert hist.max() - hist.min() <= 0.02 * hist.mean()


def test_hero_mode_converges_to_the_reference_estimator():
    """The oracle's hero-wavelength mode (four wavelengths per sample, the
    tree drawn at the hero, the hero alone with weight 4 below a hit where the
    four would sample differently) and the reference's single-wavelength
    sampler converge to the same Cornell image: 8x8-block means of independent
    frames agree within 3 sigma on X, Y and Z, and the hero mode's frames
    scatter less at the same spp."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_common import pooled_masked, primary_tie_mask
    W = H = 32
    s = scenes.cornell(W, H)
    o = O.OracleScene(s)
    frames, spp = 16, 64
    conf = _abi.make_conf(W, H, spp, 2)
    keep = ~primary_tie_mask(o, s.camera, W, H)

    def run(spectral, seed):
        out = []
        for k in range(frames):
            f, _, _ = o.render(conf, s.camera, rng=O.RNG_KEYED, seed=seed + k, prune=True,
                               spectral=spectral)
            assert np.all(np.isfinite(f))
            out.append(pooled_masked(f, keep, 8))
        return np.stack(out)

    a, b = run(O.SPECTRAL_REFERENCE, 0), run(O.SPECTRAL_HERO, 500)
    se = np.sqrt(a.var(0, ddof=1) / frames + b.var(0, ddof=1) / frames) + 1e-12
    z = np.abs(a.mean(0) - b.mean(0)) / se
    assert (z > 3.5).sum() <= 1, z.max()
    assert float(b.var(0, ddof=1).mean()) < 0.7 * float(a.var(0, ddof=1).mean())


@pytest.mark.parametrize("spectral", [O.SPECTRAL_REFERENCE, O.SPECTRAL_HERO])
def test_roulette_keeps_the_expectation_and_traces_fewer_rays(spectral):
    """Russian roulette from the second hit on (an option beyond the
    reference): the Cornell room at depth 6 converges to the same image with
    fewer closest-hit rays."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_common import pooled_masked, primary_tie_mask
    W = H = 32
    s = scenes.cornell(W, H)
    o = O.OracleScene(s)
    frames, spp = 12, 64
    conf = _abi.make_conf(W, H, spp, 6)
    keep = ~primary_tie_mask(o, s.camera, W, H)

    def run(rr, seed):
        out, rays = [], 0
        for k in range(frames):
            f, _, st = o.render(conf, s.camera, rng=O.RNG_KEYED, seed=seed + k, prune=True,
                                spectral=spectral, roulette=rr)
            out.append(pooled_masked(f, keep, 8))
            rays += int(st[0])
        return np.stack(out), rays

    (a, ra), (b, rb) = run(0, 0), run(2, 700)
    se = np.sqrt(a.var(0, ddof=1) / frames + b.var(0, ddof=1) / frames) + 1e-12
    z = np.abs(a.mean(0) - b.mean(0)) / se
    assert (z > 3.5).sum() <= 1, z.max()
    assert rb < 0.9 * ra
