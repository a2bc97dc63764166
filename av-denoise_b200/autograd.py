"""A thin torch.autograd harness over the windowed NLMeans forward (`avd_nlm_window`) and its
hand-written adjoint (`avd_nlm_backward`), and Monte-Carlo SURE for picking the strength per scene.

`NlmWindow.apply(window, strength, d, a, s)` maps a (2d+1, H, W[, C]) f32 CUDA window (normalised
samples, oldest frame first) and a 0-d f32 strength tensor to the denoised centre frame; backward
returns dL/d(window) and dL/d(strength). Everything runs in the library's kernels; this module only
moves pointers.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _abi


def _stream() -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _args(window: torch.Tensor, d: int, a: int, s: int, strength: float, self_weight: float, pair_offset: float,
          spatial_offset: float) -> _abi.AvdNlmBackward:
    frames, h, w = window.shape[:3]
    c = window.shape[3] if window.dim() == 4 else 1
    if frames != 2 * d + 1:
        raise ValueError(f"a window of temporal radius {d} holds {2 * d + 1} frames, got {frames}")
    p = _abi.AvdNlmBackward()
    p.window = window.data_ptr()
    p.width, p.height, p.channels = w, h, c
    p.temporal_radius, p.search_radius, p.patch_radius = d, a, s
    p.strength, p.self_weight, p.pair_offset, p.spatial_offset = strength, self_weight, pair_offset, spatial_offset
    return p


class NlmWindow(torch.autograd.Function):
    @staticmethod
    def forward(ctx, window, strength, d, a, s, self_weight=1.0, pair_offset=0.0, spatial_offset=0.0):
        lib = _abi.load()
        window = window.contiguous()
        if not window.is_cuda or window.dtype != torch.float32:
            raise TypeError("the window must be a float32 CUDA tensor")
        st = float(strength)
        p = _args(window, d, a, s, st, self_weight, pair_offset, spatial_offset)
        out = torch.empty(window.shape[1:], dtype=torch.float32, device=window.device)
        scratch = torch.empty(lib.avd_nlm_window_scratch_bytes(a) // 4 + 1, dtype=torch.float32,
                              device=window.device)
        p.grad_out, p.scratch = out.data_ptr(), scratch.data_ptr()
        code = lib.avd_nlm_window(C.byref(p), _stream())
        if code != 0:
            raise RuntimeError(lib.avd_last_error().decode())
        ctx.save_for_backward(window)
        ctx.params = (d, a, s, st, self_weight, pair_offset, spatial_offset)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        lib = _abi.load()
        (window,) = ctx.saved_tensors
        d, a, s, st, self_weight, pair_offset, spatial_offset = ctx.params
        p = _args(window, d, a, s, st, self_weight, pair_offset, spatial_offset)
        grad_out = grad_out.contiguous().to(torch.float32)
        grad_window = torch.empty_like(window)
        grad_strength = torch.zeros(1, dtype=torch.float32, device=window.device)
        h, w = window.shape[1:3]
        scratch = torch.empty(lib.avd_nlm_backward_scratch_bytes(w, h) // 4, dtype=torch.float32,
                              device=window.device)
        p.grad_out, p.grad_window, p.grad_strength = grad_out.data_ptr(), grad_window.data_ptr(), \
            grad_strength.data_ptr()
        p.scratch = scratch.data_ptr()
        code = lib.avd_nlm_backward(C.byref(p), _stream())
        if code != 0:
            raise RuntimeError(lib.avd_last_error().decode())
        return grad_window, grad_strength.reshape(()), None, None, None, None, None, None


def sure(window: torch.Tensor, strength: torch.Tensor, sigma: float, d: int, a: int, s: int, probes: int = 16,
         eps_scale: float = 1e-3, generator: torch.Generator | None = None) -> torch.Tensor:
    """Monte-Carlo SURE of the centre frame's denoised output: ||y - f(y)||^2 / n - sigma^2 +
    2 sigma^2 / n * div f(y), the divergence over the centre frame estimated with Rademacher probes b
    as b . (f(y + eps b) - f(y)) / eps, eps = eps_scale * sigma. Differentiable in `strength`."""
    y = window[d]
    n = y.numel()
    fy = NlmWindow.apply(window, strength, d, a, s)
    eps = eps_scale * sigma
    div = torch.zeros((), device=window.device)
    for _ in range(probes):
        b = torch.randint(0, 2, y.shape, generator=generator, device=window.device).to(torch.float32) * 2 - 1
        shifted = window.clone()
        shifted[d] = y + eps * b
        div = div + (b * (NlmWindow.apply(shifted, strength, d, a, s) - fy)).sum() / eps
    div = div / probes
    return ((y - fy) ** 2).sum() / n - sigma ** 2 + 2 * sigma ** 2 * div / n
