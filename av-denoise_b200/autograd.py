"""A thin torch.autograd harness over the windowed NLMeans forward (`avd_nlm_window`) and its
hand-written adjoint (`avd_nlm_backward`), the NL4D collab pass (`avd_collab_pass`) and its adjoint
(`avd_collab_adjoint`), and Monte-Carlo SURE for picking the strength per scene.

`NlmWindow.apply(window, strength, d, a, s)` maps a (2d+1, H, W[, C]) f32 CUDA window (normalised
samples, oldest frame first) and a 0-d f32 strength tensor to the denoised centre frame; backward
returns dL/d(window) and dL/d(strength).

`Nl4dPass.apply(window, sigma, config)` maps a (2d+1, H, W, C) f32 CUDA window (C = 1 or 2) and a
(C,) f32 noise-level tensor to the centre frame one collab pass denoises (its accumulators'
A / W); backward returns dL/d(window) and dL/d(sigma) with the pass's groups and keep decisions
held fixed. Everything runs in the library's kernels; this module only moves pointers.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np
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


@dataclass(frozen=True)
class Nl4dPassConfig:
    """One collab pass's settings (collab/kernels/fused/mod.rs:170-234 names them): the window's
    temporal radius, the centre search radius, the trajectory refine, the threshold (pooled when
    `pool_ratio` is set), the Kaiser taper, the DCT noise correlation `rho`, the Wiener stage, and
    the motion of each neighbour (`mv_field` i32 (dx, dy) per 8-step block of 16x16 blocks,
    `confidence` f32 per block; neighbours ordered d-1, d+1, d-2, d+2, ...; zero motion at full
    confidence when None)."""

    radius: int = 1
    spatial_radius: int = 5
    refine: int = 2
    lambda_ht: float = 2.7
    pool_ratio: Optional[float] = None
    kaiser_beta: float = 2.0
    rho: float = 0.0
    c_min: float = 0.05
    wiener: bool = False
    mv_field: Optional[torch.Tensor] = None
    confidence: Optional[torch.Tensor] = None


class _Nl4dState:
    """The device buffers one pass and its adjoint share."""

    BLKSIZE, BLK_STEP = 16, 8

    def __init__(self, window: torch.Tensor, sigma: torch.Tensor, cfg: Nl4dPassConfig):
        lib = _abi.load()
        frames, h, w, c = window.shape
        if frames != 2 * cfg.radius + 1 or c not in (1, 2):
            raise ValueError("the window holds 2 radius + 1 frames of 1 or 2 channels")
        dev = window.device
        self.shape = (frames, h, w, c)
        prof = (C.c_float * 8)()
        lib.avd_dct_noise_profile(cfg.rho, prof)
        kai = (C.c_float * 8)()
        lib.avd_kaiser_window(cfg.kaiser_beta, kai)
        self.profile = torch.tensor(list(prof), dtype=torch.float32, device=dev)
        self.kaiser = torch.tensor(list(kai), dtype=torch.float32, device=dev)
        sig = sigma.detach().to(torch.float32).reshape(-1)
        if sig.numel() != c:
            raise ValueError("one noise level per channel")
        # The weight-scale word, aggregate.rs:79-99 (sigma_0^2 g_max^2, floored at 1e-12); the adjoint
        # reads it as proportional to sigma_0^2.
        f = np.float32
        g, s0 = f(max(prof)), f(float(sig[0]))
        ws = ((s0 * s0) * g) * g
        ws = float(ws) if np.isfinite(ws) and ws > f(1e-12) else 1e-12
        self.noise = torch.cat([sig, torch.tensor([ws, 0.0], device=dev)]).contiguous()
        bx, by = -(-w // self.BLK_STEP), -(-h // self.BLK_STEP)
        neighbours = 2 * cfg.radius
        self.mv = (cfg.mv_field if cfg.mv_field is not None else
                   torch.zeros(max(neighbours, 1) * bx * by * 2, dtype=torch.int32, device=dev)).contiguous()
        self.conf = (cfg.confidence if cfg.confidence is not None else
                     torch.ones(max(neighbours, 1) * bx * by, dtype=torch.float32, device=dev)).contiguous()
        order = [s for t in range(cfg.radius) for s in (cfg.radius - 1 - t, cfg.radius + 1 + t)]
        self.slots = torch.tensor(order or [0], dtype=torch.int32, device=dev)
        self.curve = torch.zeros(16, dtype=torch.float32, device=dev)
        self.accum = torch.zeros(frames * h * w * c, dtype=torch.int32, device=dev)
        self.wsum = torch.zeros(frames * h * w, dtype=torch.int32, device=dev)
        self.refs = lib.avd_collab_refs(w, h)
        self.group_weight = torch.zeros(self.refs, dtype=torch.float32, device=dev)
        self.members = torch.zeros(lib.avd_collab_member_bytes(w, h) // 4, dtype=torch.int32, device=dev)
        p = _abi.AvdCollabPass()
        p.ring, p.mv_field, p.confidence = window.data_ptr(), self.mv.data_ptr(), self.conf.data_ptr()
        p.neighbour_slots, p.noise, p.noise_curve = self.slots.data_ptr(), self.noise.data_ptr(), self.curve.data_ptr()
        p.dct_profile, p.kaiser = self.profile.data_ptr(), self.kaiser.data_ptr()
        p.accum, p.wsum, p.group_weight = self.accum.data_ptr(), self.wsum.data_ptr(), self.group_weight.data_ptr()
        p.members = self.members.data_ptr()
        p.width, p.height, p.channels, p.centre_slot = w, h, c, cfg.radius
        p.sigma_word, p.weight_scale_word, p.curve_valid_word = 0, c, c + 1
        p.radius, p.refine, p.spatial_radius, p.k_max = cfg.radius, cfg.refine, cfg.spatial_radius, 8
        p.mv_stride, p.conf_stride = bx * by * 2, bx * by
        p.blk_step, p.blksize, p.blocks_x, p.blocks_y = self.BLK_STEP, self.BLKSIZE, bx, by
        p.pooled, p.pool_ratio = int(cfg.pool_ratio is not None), float(cfg.pool_ratio or 0.0)
        p.c_min, p.lambda_ht = cfg.c_min, cfg.lambda_ht
        p.accum_scale = lib.avd_cross_frame_accum_scale(cfg.spatial_radius, cfg.radius)
        p.wiener = int(cfg.wiener)
        self.p = p
        self.window = window

    def run(self) -> None:
        lib = _abi.load()
        code = lib.avd_collab_pass(C.byref(self.p), _stream())
        if code != 0:
            raise RuntimeError(lib.avd_last_error().decode())


class Nl4dPass(torch.autograd.Function):
    @staticmethod
    def forward(ctx, window, sigma, cfg: Nl4dPassConfig):
        window = window.contiguous()
        if not window.is_cuda or window.dtype != torch.float32 or window.dim() != 4:
            raise TypeError("the window must be a (frames, H, W, C) float32 CUDA tensor")
        st = _Nl4dState(window, sigma, cfg)
        st.run()
        frames, h, w, c = st.shape
        centre = cfg.radius
        acc = st.accum.view(frames, h, w, c)[centre].to(torch.float32)
        wsum = st.wsum.view(frames, h, w)[centre].to(torch.float32)
        covered = (wsum > 0).unsqueeze(-1)
        # collab_normalise (aggregate.rs:240-290): accum x 5 / wsum, which is A / W in real units.
        out = torch.where(covered, acc * 5.0 / torch.where(covered, wsum.unsqueeze(-1), torch.ones_like(acc)), acc)
        ctx.state = st
        ctx.save_for_backward(out)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        lib = _abi.load()
        st = ctx.state
        (out,) = ctx.saved_tensors
        frames, h, w, c = st.shape
        centre = st.p.centre_slot
        scale = st.p.accum_scale
        wsum = st.wsum.view(frames, h, w)[centre].to(torch.float32) / (5.0 * scale)  # W, real units
        covered = wsum > 0
        safe = torch.where(covered, wsum, torch.ones_like(wsum)).unsqueeze(-1)
        g = grad_out.to(torch.float32) * covered.unsqueeze(-1)
        grad_accum = torch.zeros(frames, h, w, c, dtype=torch.float32, device=out.device)
        grad_wsum = torch.zeros(frames, h, w, dtype=torch.float32, device=out.device)
        grad_accum[centre] = g / safe
        grad_wsum[centre] = -(g * out / safe).sum(-1)
        grad_window = torch.zeros_like(st.window)
        grad_refs = torch.empty(st.refs * c, dtype=torch.float32, device=out.device)
        adj = _abi.AvdCollabAdjoint(grad_accum.data_ptr(), grad_wsum.data_ptr(), grad_window.data_ptr(),
                                    grad_refs.data_ptr())
        code = lib.avd_collab_adjoint(C.byref(st.p), C.byref(adj), _stream())
        if code != 0:
            raise RuntimeError(lib.avd_last_error().decode())
        grad_sigma = grad_refs.view(st.refs, c).sum(0)
        return grad_window, grad_sigma, None


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
