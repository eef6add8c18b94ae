"""mcfftExecHost: host buffers in and out, copies and transforms pipelined
over chunks of whole transforms.  The result must match the oracle (and the
device-buffer exec of the same plan) for chunked single-shape plans of both
forms, one-chunk plans (batch 1, uneven batches), repeated calls (which
replay the chunk plan's graphs), page-locked and pageable host memory, and
in-place host buffers; overlapping buffers of different element sizes are
refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from oracle import oracle  # noqa: E402
from tests.gpu_util import compare, rand_complex, rounded, run  # noqa: E402

PLAIN_TOL = 1e-3
SPLIT_TOL = 2e-6


def host_in(x: np.ndarray, f16: bool, pinned: bool) -> torch.Tensor:
    flat = np.ascontiguousarray(x.reshape(-1))
    if f16:
        ri = np.stack([flat.real, flat.imag], -1).astype(np.float16).reshape(-1)
        t = torch.from_numpy(ri.view(np.uint16).copy())
    else:
        t = torch.from_numpy(flat.astype(np.complex64).view(np.float32).copy())
    return t.pin_memory() if pinned else t


def host_out(elements: int, f16: bool, pinned: bool) -> torch.Tensor:
    t = torch.empty(elements * 2, dtype=torch.float16 if f16 else torch.float32)
    t.view(torch.uint8).fill_(0xFF)
    return t.pin_memory() if pinned else t


def decode(t: torch.Tensor) -> np.ndarray:
    h = t.numpy().astype(np.float64)
    return h[0::2] + 1j * h[1::2]


def exec_host(plan, hin, hout, direction=mc.FORWARD):
    plan.exec_host_ptr(hin.data_ptr(), hout.data_ptr(), direction,
                       torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    plan.check_status()
    return decode(hout)


@pytest.mark.parametrize("pinned", [True, False])
def test_plain_chunked_matches_oracle_and_device_exec(monkeypatch, pinned):
    n, batch = 1 << 16, 32
    monkeypatch.setenv("MCFFT_HOST_CHUNK_BYTES", str(1 << 20))  # chunks of up to 4 transforms
    # The chunk plans (1, 2, 4 transforms) are tuned apart from the full
    # plan and may take another four-step split, whose FP16 roundings differ;
    # untuned, every plan takes the same split and the outputs must agree.
    monkeypatch.setenv("MCFFT_AUTOTUNE", "0")
    x = rand_complex((batch, n), seed=21)
    with mc.Plan((n,), batch, mc.PREC_FP16) as p:
        hin = host_in(x, True, pinned)
        hout = host_out(n * batch, True, pinned)
        y = exec_host(p, hin, hout)
        y_dev, sl = run(p, x, True)
        for _ in range(2):  # repeated calls replay the chunk plan's graphs
            hout.view(torch.uint8).fill_(0xFF)
            assert np.array_equal(exec_host(p, hin, hout), y)
    ref = oracle.fft1d(rounded(x, True)) * 2.0 ** sl
    rel, mx = compare(y, ref)
    assert rel < PLAIN_TOL, (rel, mx)
    assert np.max(np.abs(y - y_dev)) <= 1e-3 * np.max(np.abs(y_dev))


def test_split_f16_input_chunked(monkeypatch):
    n, batch = 4096, 48
    monkeypatch.setenv("MCFFT_HOST_CHUNK_BYTES", str(64 << 10))  # chunks of up to 4 transforms
    x = rand_complex((batch, n), seed=22)
    with mc.Plan((n,), batch, mc.PREC_SPLIT, mc.FLAG_INPUT_F16) as p:
        assert p.info().scale_log2 == 0
        y = exec_host(p, host_in(x, True, True), host_out(n * batch, False, True))
        yi = exec_host(p, host_in(x, True, True), host_out(n * batch, False, True), mc.INVERSE)
    ref = oracle.fft1d(rounded(x, True))
    rel, _ = compare(y, ref)
    assert rel < SPLIT_TOL, rel
    refi = oracle.fft1d(rounded(x, True), sign=1)
    reli, _ = compare(yi, refi)
    assert reli < SPLIT_TOL, reli


def test_2d_chunked(monkeypatch):
    nx, ny, batch = 128, 256, 6
    monkeypatch.setenv("MCFFT_HOST_CHUNK_BYTES", str(256 << 10))  # chunks of up to 2 transforms
    x = rand_complex((batch, nx, ny), seed=23)
    with mc.Plan((nx, ny), batch, mc.PREC_FP16) as p:
        sl = p.info().scale_log2
        y = exec_host(p, host_in(x, True, True), host_out(nx * ny * batch, True, True))
    ref = oracle.fftnd(rounded(x, True), (nx, ny)) * 2.0 ** sl
    rel, _ = compare(y, ref)
    assert rel < PLAIN_TOL, rel


def test_one_chunk_plans():
    # batch 1: one chunk, no chunk plan
    n = 1 << 18
    x = rand_complex((1, n), seed=24)
    with mc.Plan((n,), 1, mc.PREC_FP16) as p:
        y = exec_host(p, host_in(x, True, True), host_out(n, True, True))
        y_dev, sl = run(p, x, True)
    assert np.array_equal(y, y_dev)
    # uneven batch (batch queue): one chunk through the plan itself
    descs, off = [], 0
    for shape in ((256,), (8192,), (8192,), (128, 256)):
        nn = int(np.prod(shape))
        descs.append((shape, 1, off, off))
        off += nn
    xb = rand_complex((off,), seed=25)
    with mc.Plan(descs=descs, precision=mc.PREC_FP16) as p:
        yb = exec_host(p, host_in(xb, True, True), host_out(off, True, True))
        yb_dev, _ = run(p, xb, True)
    assert np.array_equal(yb, yb_dev)


def test_in_place_host_buffer(monkeypatch):
    n, batch = 8192, 16
    monkeypatch.setenv("MCFFT_HOST_CHUNK_BYTES", str(64 << 10))  # chunks of up to 2 transforms
    x = rand_complex((batch, n), seed=26)
    with mc.Plan((n,), batch, mc.PREC_FP16) as p:
        buf = host_in(x, True, True)
        y_sep = exec_host(p, buf, host_out(n * batch, True, True))
        p.exec_host_ptr(buf.data_ptr(), buf.data_ptr(), mc.FORWARD,
                        torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        p.check_status()
        hb = buf.view(torch.float16).numpy().astype(np.float64)
        assert np.array_equal(hb[0::2] + 1j * hb[1::2], y_sep)


def test_overlap_of_unequal_elements_refused():
    n, batch = 4096, 8
    with mc.Plan((n,), batch, mc.PREC_SPLIT, mc.FLAG_INPUT_F16) as p:
        buf = torch.zeros(n * batch * 4, dtype=torch.float32).pin_memory()
        with pytest.raises(mc.McfftError) as ei:
            p.exec_host_ptr(buf.data_ptr(), buf.data_ptr(), mc.FORWARD, 0)
        assert ei.value.code == mc.INVALID_VALUE
