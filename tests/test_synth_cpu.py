"""Synthetic workload builders (cel_v3_b200/synth.py)."""
import numpy as np
import torch

from cel_v3_b200 import synth


def test_device_assembly_equals_host_assembly():
    """The torch assembly (run here on the CPU) equals the host assembly bit
    for bit."""
    for grid in [(5, 4, 3), (7, 6, 9), (1, 1, 4), (3, 1, 1)]:
        g, (kx, ky, kz) = synth.lognormal_faces(np.random.default_rng(1), *grid)
        rp, ci, v = synth.diffusion7(*grid, kx, ky, kz)
        r2, c2, v2 = synth.diffusion7_device(*grid, np.exp(g), device="cpu")
        assert np.array_equal(rp, r2.numpy()) and np.array_equal(ci, c2.numpy())
        assert np.array_equal(v, v2.numpy())


def test_differentiation_problems_draw_order():
    p = synth.differentiation_problems(side=6, batch=3)
    cx, cy, cz = synth.face_counts(6, 6, 6)
    r6, r7 = np.random.default_rng(6), np.random.default_rng(7)
    for g, b, xt in p:
        assert np.array_equal(g, r6.standard_normal(cx + cy + cz))
        assert np.array_equal(b, r7.uniform(-1.0, 1.0, 216))
        assert np.array_equal(xt, r7.random(216))
