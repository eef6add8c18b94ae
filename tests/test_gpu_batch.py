"""Uneven batches: many transforms of different lengths and dimensionality
in one plan (mcfftPlanCreateBatch), run by the persistent batch kernel in
one launch, each transform checked against the FP64 oracle -- with the
transforms of one shape next to each other, and in any order (one
descriptor per transform, shapes interleaved, input and output orders
different: per-transform coordinate tables and row gathers).  Also the
batch kernel forced onto single-shape plans (MCFFT_QUEUE=1), including the
four-step 1D and 2D/3D dependency chains.

Tolerances as in test_gpu_parity: plain rel-L2 <= 1e-3, split <= 2e-6.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from oracle import oracle  # noqa: E402
from tests.gpu_util import compare, from_device, rand_complex, rounded, to_device  # noqa: E402

PLAIN_TOL = 1e-3
SPLIT_TOL = 2e-6

# (shape, count): 1D single-pass and four-step lengths, 2D and 3D shapes
SHAPES = [((256,), 5), ((1024,), 3), ((4096,), 2), ((8192,), 1), ((1 << 16,), 1),
          ((128, 256), 2), ((512, 128), 1), ((64, 32, 128), 1)]


def _layout(shapes, gap):
    """One descriptor per transform, laid out in order with `gap` elements
    between groups of one shape; returns descs and the total length."""
    descs, off = [], 0
    for shape, count in shapes:
        n = int(np.prod(shape))
        for _ in range(count):
            descs.append((shape, 1, off, off))
            off += n
        off += gap
    return descs, off


def _run_batch(descs, total, precision, flags=mc.FLAG_NONE, seed=7):
    f16 = precision == mc.PREC_FP16 or bool(flags & mc.FLAG_INPUT_F16)
    x = rand_complex((total,), seed=seed)
    xd = to_device(x, f16)
    odt = torch.complex64 if precision == mc.PREC_SPLIT else torch.complex32
    out = torch.empty(total, dtype=odt, device="cuda")
    out.view(torch.uint8).fill_(0xFF)
    with mc.Plan(descs=descs, precision=precision, flags=flags) as p:
        info = p.info()
        p.exec_ptr(xd.data_ptr(), out.data_ptr(), mc.FORWARD, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        p.check_status()
    return rounded(x, f16), from_device(out), info


def _check_each(descs, xr, y, plain):
    worst = 0.0
    for shape, batch, io, oo in descs:
        n = int(np.prod(shape))
        ref = oracle.fftnd(xr[io:io + n * batch].reshape((batch,) + tuple(shape)), shape)
        if plain:
            ref = ref * 2.0 ** -int(np.log2(n))
        rel, _ = compare(y[oo:oo + n * batch], ref)
        worst = max(worst, rel)
    return worst


@pytest.mark.parametrize("gap", [0, 64])
def test_uneven_batch_plain_one_launch(gap):
    descs, total = _layout(SHAPES, gap)
    xr, y, info = _run_batch(descs, total, mc.PREC_FP16)
    assert info.launches == 1, info.launches
    assert _check_each(descs, xr, y, True) < PLAIN_TOL
    if gap:
        # gaps between shape groups are never written
        assert np.isnan(y[int(np.prod(SHAPES[0][0])) * SHAPES[0][1]])


@pytest.mark.parametrize("flags", [mc.FLAG_INPUT_F16, mc.FLAG_NONE])
def test_uneven_batch_split_one_launch(flags):
    descs, total = _layout(SHAPES, 0)
    xr, y, info = _run_batch(descs, total, mc.PREC_SPLIT, flags)
    assert info.launches == 1, info.launches
    assert _check_each(descs, xr, y, False) < SPLIT_TOL


@pytest.mark.parametrize("shape,batch", [((1 << 20,), 2), ((4096,), 8), ((1024, 1024), 1),
                                         ((32, 64, 256), 2)])
def test_queue_forced_single_shape_split(shape, batch, monkeypatch):
    monkeypatch.setenv("MCFFT_QUEUE", "1")
    n = int(np.prod(shape))
    descs = [(shape, batch, 0, 0)]
    xr, y, info = _run_batch(descs, n * batch, mc.PREC_SPLIT, mc.FLAG_INPUT_F16, seed=n)
    assert info.launches == 1
    assert _check_each(descs, xr, y, False) < SPLIT_TOL


@pytest.mark.parametrize("shape,batch", [((1 << 20,), 2), ((1 << 14,), 8), ((1024, 1024), 2),
                                         ((256, 512), 3), ((32, 64, 256), 2), ((128, 64, 64), 1)])
def test_queue_forced_single_shape(shape, batch, monkeypatch):
    monkeypatch.setenv("MCFFT_QUEUE", "1")
    n = int(np.prod(shape))
    descs = [(shape, batch, 0, 0)]
    xr, y, info = _run_batch(descs, n * batch, mc.PREC_FP16, seed=n)
    assert info.launches == 1
    assert _check_each(descs, xr, y, True) < PLAIN_TOL


def test_uneven_batch_8k_tiles_stays_one_launch(monkeypatch):
    # 8K-point tiles forced: every pass the batch kernel holds in 8K takes
    # it (the batch kernel's 16-warp 8K routines); L = 4096 keeps 16K tiles,
    # the only shape the batch kernel holds for it, so the plan stays one launch
    monkeypatch.setenv("MCFFT_TILE_POINTS", "8192")
    monkeypatch.setenv("MCFFT_AUTOTUNE", "0")
    descs, total = _layout(SHAPES, 0)
    xr, y, info = _run_batch(descs, total, mc.PREC_FP16, seed=9)
    assert info.launches == 1, info.launches
    assert _check_each(descs, xr, y, True) < PLAIN_TOL


def test_queue_repeated_exec_and_inverse():
    # counters are reset per exec; the inverse direction uses the conjugate tables
    descs, total = _layout(SHAPES[:6], 0)
    x = rand_complex((total,), seed=11)
    xd = to_device(x, True)
    out = torch.empty(total, dtype=torch.complex32, device="cuda")
    with mc.Plan(descs=descs, precision=mc.PREC_FP16) as p:
        for direction in (mc.FORWARD, mc.INVERSE, mc.FORWARD):
            out.view(torch.uint8).fill_(0xFF)
            p.exec_ptr(xd.data_ptr(), out.data_ptr(), direction, torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            p.check_status()
            y = from_device(out)
            xr = rounded(x, True)
            for shape, batch, io, oo in descs:
                n = int(np.prod(shape))
                ref = oracle.fftnd(xr[io:io + n].reshape((1,) + tuple(shape)), shape, sign=direction)
                rel, _ = compare(y[oo:oo + n], ref * 2.0 ** -int(np.log2(n)))
                assert rel < PLAIN_TOL, (shape, direction, rel)


def _scattered(shapes, seed):
    """One descriptor per transform; the transforms lie in a seeded random
    order in the input and in another in the output."""
    items = [shape for shape, count in shapes for _ in range(count)]
    rng = np.random.default_rng(seed)
    sizes = [int(np.prod(sh)) for sh in items]

    def place(order):
        offs, off = [0] * len(items), 0
        for i in order:
            offs[i] = off
            off += sizes[i]
        return offs, off

    ioffs, total = place(rng.permutation(len(items)))
    ooffs, _ = place(rng.permutation(len(items)))
    return [(sh, 1, io, oo) for sh, io, oo in zip(items, ioffs, ooffs)], total


@pytest.mark.parametrize("prec,flags", [(mc.PREC_FP16, mc.FLAG_NONE),
                                        (mc.PREC_SPLIT, mc.FLAG_INPUT_F16),
                                        (mc.PREC_SPLIT, mc.FLAG_NONE)])
@pytest.mark.parametrize("seed", [1, 2])
def test_uneven_batch_any_order_one_launch(prec, flags, seed):
    shapes = SHAPES + [((256,), 7), ((1024,), 5), ((128, 256), 2)]
    descs, total = _scattered(shapes, seed)
    xr, y, info = _run_batch(descs, total, prec, flags, seed=seed)
    assert info.launches == 1, info.launches
    plain = prec == mc.PREC_FP16
    assert _check_each(descs, xr, y, plain) < (PLAIN_TOL if plain else SPLIT_TOL)


def test_uneven_batch_any_order_3d_and_repeat():
    """3D transforms interleaved with others (the middle pass's per-slab
    table), executed twice (the counters and tables are reused)."""
    shapes = [((32, 64, 128), 2), ((64, 32, 32), 3), ((4096,), 3), ((1 << 15,), 2)]
    descs, total = _scattered(shapes, 5)
    x = rand_complex((total,), seed=5)
    xd = to_device(x, True)
    out = torch.empty(total, dtype=torch.complex32, device="cuda")
    with mc.Plan(descs=descs, precision=mc.PREC_FP16) as p:
        assert p.info().launches == 1
        for _ in range(2):
            out.view(torch.uint8).fill_(0xFF)
            p.exec_ptr(xd.data_ptr(), out.data_ptr(), mc.FORWARD, torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            p.check_status()
            assert _check_each(descs, rounded(x, True), from_device(out), True) < PLAIN_TOL
