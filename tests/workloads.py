"""The stated benchmark configurations and their seeded synthetic inputs,
shared by the GPU parity tests and bench.py.

Each input is drawn in float64 with numpy's PCG64 generator and rounded
once to the storage type (FP16 or FP32) by the caller; the FP64 oracle then
sees exactly what the GPU sees.  No public dataset is involved.

  c1  1D N=4096, batch 256, re/im uniform [-1, 1), seed 0
  c2  1D N=2^20, batch 64, re/im uniform [-1, 1), seed 1
  c3  2D 1024 x 1024, batch 16, seed 2: uniform [-1, 1) re/im, and a
      wide-range variant with |z| log-uniform in [1e-3, 1e3], phase uniform
  c4  3D 256^3, batch 1, seed 3: eight plane waves (integer wave vectors in
      [-64, 64]^3, real amplitudes uniform [0, 1)) plus complex Gaussian
      noise of standard deviation 1e-2 per component
  c5  uneven batch, seed 4: 4096 1D transforms with N = 2^e, e uniform in
      8..16, plus 64 2D transforms with sides uniform in {128, 256, 512};
      re/im uniform [-1, 1)
"""
from __future__ import annotations

import numpy as np

CONFIGS = {
    # name: (dims, batch, seed, description)
    "c1": ((4096,), 256, 0, "1D N=4096 batch 256"),
    "c2": ((1 << 20,), 64, 1, "1D N=2^20 batch 64"),
    "c3": ((1024, 1024), 16, 2, "2D 1024x1024 batch 16"),
    "c4": ((256, 256, 256), 1, 3, "3D 256^3 batch 1"),
}


def uniform(shape, seed):
    """re, im uniform in [-1, 1) (re first, then im)."""
    rng = np.random.default_rng(seed)
    re = rng.uniform(-1, 1, shape)
    im = rng.uniform(-1, 1, shape)
    return re + 1j * im


def wide_range(shape, seed):
    """|z| log-uniform in [1e-3, 1e3], phase uniform in [0, 2 pi)."""
    rng = np.random.default_rng(seed)
    mag = 10.0 ** rng.uniform(-3, 3, shape)
    ph = rng.uniform(0, 2 * np.pi, shape)
    return mag * np.exp(1j * ph)


def plane_waves(n=256, waves=8, sigma=1e-2, seed=3):
    """c4's input, shape (1, n, n, n): sum over p of a_p exp(2 pi i k_p . r / n)
    with k_p integer in [-64, 64]^3 and a_p uniform [0, 1) (real), plus
    complex Gaussian noise N(0, sigma^2) per component."""
    rng = np.random.default_rng(seed)
    k = rng.integers(-64, 65, (waves, 3))
    a = rng.uniform(0, 1, waves)
    r = np.arange(n)
    x = np.zeros((n, n, n), np.complex128)
    for p in range(waves):
        ex = np.exp(2j * np.pi * k[p, 0] * r / n)
        ey = np.exp(2j * np.pi * k[p, 1] * r / n)
        ez = np.exp(2j * np.pi * k[p, 2] * r / n)
        x += a[p] * ex[:, None, None] * (ey[:, None] * ez[None, :])[None, :, :]
    x += rng.normal(0, sigma, (n, n, n)) + 1j * rng.normal(0, sigma, (n, n, n))
    return x.reshape(1, n, n, n)


def uneven_shapes(seed=4):
    """c5's transforms in the order they are drawn: 4096 1D lengths 2^e
    (e uniform in 8..16), then 64 2D shapes (sides uniform in {128, 256,
    512})."""
    rng = np.random.default_rng(seed)
    e = rng.integers(8, 17, 4096)
    sides = np.array([128, 256, 512])
    nx = sides[rng.integers(0, 3, 64)]
    ny = sides[rng.integers(0, 3, 64)]
    return [(1 << int(v),) for v in e] + [(int(a), int(b)) for a, b in zip(nx, ny)]


def uneven_layout(order="draw", seed=4):
    """c5's descriptors, one per transform, packed back to back in the given
    order: "draw" (as drawn), "sorted" (by dimensionality, then shape) or
    "shuffled" (a seeded permutation of the draw).  Returns (shapes,
    offsets, total elements)."""
    shapes = uneven_shapes(seed)
    if order == "sorted":
        shapes = sorted(shapes, key=lambda s: (len(s), s))
    elif order == "shuffled":
        perm = np.random.default_rng(seed + 1000).permutation(len(shapes))
        shapes = [shapes[i] for i in perm]
    elif order != "draw":
        raise ValueError(order)
    offs, off = [], 0
    for s in shapes:
        offs.append(off)
        off += int(np.prod(s))
    return shapes, offs, off


def uneven_input(total, seed=4):
    """c5's input values: re/im uniform [-1, 1), interleaved, as complex."""
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1, 1, 2 * total)
    return v[0::2] + 1j * v[1::2]


def flops_5nlogn(dims, batch=1):
    n = int(np.prod(dims))
    return 5.0 * n * np.log2(n) * batch
