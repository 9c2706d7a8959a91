"""The GGX masking term's tangent: the kernels evaluate tan(acos(c)) as
sqrt(1 - c^2) / c (`tanOfAcos` in csrc/cg_device.cuh), the reference and the
oracle as tan(acos(c)) (shading/dist/rough_reflection.wesl).  On the cosines
the kernels pass (c >= 1e-6) the two agree to a few float32 rounding steps,
and both are NaN for a cosine a rounding step above 1, which is where the
reference's NaN samples come from."""
import numpy as np


def _identity_f32(c):
    c = c.astype(np.float32)
    one_minus = np.float32(1.0) - c.astype(np.float64) * c  # fmaf(-c, c, 1): one rounding
    with np.errstate(invalid="ignore"):
        return (np.sqrt(one_minus.astype(np.float32)) / c).astype(np.float32)


def test_identity_matches_tan_of_acos():
    rng = np.random.default_rng(7)
    c = np.concatenate([np.float32(10.0) ** rng.uniform(-6, 0, 200_000).astype(np.float32),
                        np.float32(1.0) - np.float32(10.0) ** rng.uniform(-7, -1, 50_000).astype(np.float32),
                        np.array([1e-6, 0.5, 1.0], np.float32)]).astype(np.float32)
    c = np.clip(c, np.float32(1e-6), np.float32(1.0))
    exact = np.tan(np.arccos(c.astype(np.float64)))
    got = _identity_f32(c).astype(np.float64)
    ref32 = np.tan(np.arccos(c)).astype(np.float64)  # the reference's form in float32
    rel_got = np.abs(got - exact) / np.maximum(np.abs(exact), 1e-30)
    rel_ref = np.abs(ref32 - exact) / np.maximum(np.abs(exact), 1e-30)
    # the identity is at least as close to the exact value as the float32
    # tan(acos(c)) chain, up to a few rounding steps
    assert float(np.max(rel_got)) < 4e-7
    assert float(np.quantile(rel_got, 0.999)) <= float(np.quantile(rel_ref, 0.999)) + 4e-7
    assert got[-1] == 0.0  # c = 1


def test_identity_is_nan_above_one_like_acos():
    above = np.nextafter(np.float32(1.0), np.float32(2.0), dtype=np.float32)
    c = np.array([above, np.float32(1.0000005), np.float32(1.5)], np.float32)
    with np.errstate(invalid="ignore"):
        assert np.all(np.isnan(np.arccos(c)))
    assert np.all(np.isnan(_identity_f32(c)))
