"""Helpers for the GPU parity tests: run a plan through the C ABI on torch
buffers and compare with the FP64 oracle on the same (storage-rounded)
inputs."""
import numpy as np
import torch

import mcfft_b200 as mc
from oracle import oracle


def rand_complex(shape, seed, dist="uniform"):
    rng = np.random.default_rng(seed)
    if dist == "uniform":
        return rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)
    if dist == "wide":
        mag = 10.0 ** rng.uniform(-3, 3, shape)
        ph = rng.uniform(0, 2 * np.pi, shape)
        return mag * np.exp(1j * ph)
    raise ValueError(dist)


def to_device(x: np.ndarray, f16: bool) -> torch.Tensor:
    """complex128 numpy -> device complex32 (f16) or complex64 tensor, flat."""
    flat = np.ascontiguousarray(x.reshape(-1))
    if f16:
        ri = np.stack([flat.real, flat.imag], -1).astype(np.float16)
        t = torch.from_numpy(ri.reshape(-1).view(np.uint16).copy()).cuda()
        return t.view(torch.complex32)
    return torch.from_numpy(flat.astype(np.complex64)).cuda()


def from_device(t: torch.Tensor) -> np.ndarray:
    if t.dtype == torch.complex32:
        h = t.view(torch.uint16).cpu().numpy().view(np.float16).astype(np.float64)
        return h[0::2] + 1j * h[1::2]
    return t.cpu().numpy().astype(np.complex128)


def rounded(x: np.ndarray, f16: bool) -> np.ndarray:
    """The value the device actually sees after storage rounding."""
    if f16:
        return (x.real.astype(np.float16).astype(np.float64)
                + 1j * x.imag.astype(np.float16).astype(np.float64))
    return x.astype(np.complex64).astype(np.complex128)


def run(plan: mc.Plan, x: np.ndarray, in_f16: bool, direction=mc.FORWARD):
    """Exec the plan on x; returns (output as complex128, scale_log2)."""
    xd = to_device(x, in_f16)
    info = plan.info()
    out_dtype = torch.complex64 if plan.precision == mc.PREC_SPLIT else torch.complex32
    out = torch.empty(info.elements, dtype=out_dtype, device="cuda")
    out.view(torch.uint8).fill_(0xFF)  # NaN poison: every output must be written
    plan.exec_ptr(xd.data_ptr(), out.data_ptr(), direction,
                  torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    plan.check_status()
    return from_device(out), info.scale_log2


def compare(y: np.ndarray, ref: np.ndarray):
    return oracle.error_norms(y.reshape(-1), ref.reshape(-1))
