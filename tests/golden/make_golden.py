"""Generates the golden alias-table fixtures from the reference itself.

Runs the reference's own AliasTable (src/pathtracing/alias_table.h of
ray847/CrystalGraphics, compiled unmodified by `make -C oracle ref` into
oracle/_ref/libref_alias.so) on seeded weight vectors and stores weights and
entries in tests/golden/alias_tables.npz.  Needs the reference tree; the
fixtures it writes are committed so tests run without it.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402


def weight_sets():
    rng = np.random.default_rng(1234)
    yield "probe", np.array([1.0, 2.0, 3.0, 4.0])
    yield "single", np.array([0.7])
    yield "uniform64", np.full(64, 1.0 / 64)
    yield "zeros", np.zeros(5)
    yield "with_zero", np.array([0.0, 1.0, 0.0, 2.5, 0.0])
    yield "negative", np.array([-1.0, 2.0, 3.0])
    yield "loguniform64", np.exp(rng.uniform(np.log(1.0), np.log(100.0), 64))
    yield "lognormal10k", np.exp(rng.normal(0.0, 2.0, 10_000))
    w = np.exp(rng.normal(0.0, 2.0, 10_000)).astype(np.float32)
    yield "lognormal10k_f32norm", (w / w.sum(dtype=np.float32)).astype(np.float32).astype(np.float64)
    yield "ragged7", np.array([1e-30, 1.0, 1e30, 3.0, 0.5, 1e-5, 7.0])


def main():
    oracle.build(reference=True)
    if not oracle.ref_alias_available():
        raise SystemExit("reference tree not available: cannot generate fixtures")
    out = {}
    for name, w in weight_sets():
        e = oracle.ref_alias_build(w)
        out[f"{name}__w"] = np.asarray(w, np.float64)
        out[f"{name}__alias"] = e["alias"].copy()
        out[f"{name}__prob"] = e["prob"].copy()
    np.savez_compressed(os.path.join(HERE, "alias_tables.npz"), **out)
    print("wrote", len(out) // 3, "tables")


if __name__ == "__main__":
    main()
