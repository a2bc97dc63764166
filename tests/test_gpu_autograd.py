"""The torch.autograd harness over the NLMeans forward and adjoint, and SURE-driven strength
selection on a 128x128 crop (1080p-generator content, 10-bit luma, sigma = 16 codes, d=2 a=5 s=2,
16 Rademacher probes, eps = 1e-3 sigma, Adam on log strength)."""

import numpy as np
import pytest

from test_oracle_nlm_backward import frames_for

pytestmark = pytest.mark.gpu


def test_autograd_gradients_match_the_fp64_adjoint(oracle):
    import torch

    from av_denoise_b200.autograd import NlmWindow

    d, a, s, strength = 1, 3, 1, 6.0
    window = frames_for(3, 48, 40, 1, 2 * d + 1)
    g = np.random.default_rng(1).normal(0, 1, (40, 48, 1))
    win = torch.from_numpy(np.stack(window)[..., 0].copy()).cuda().requires_grad_(True)
    st = torch.tensor(strength, device="cuda", requires_grad=True)
    out = NlmWindow.apply(win, st, d, a, s)
    (out * torch.from_numpy(g[..., 0]).float().cuda()).sum().backward()
    want, want_s = oracle.nlm_backward(window, d, a, s, strength, g)
    got = win.grad.cpu().numpy()
    rel = np.linalg.norm(got - want[..., 0]) / np.linalg.norm(want)
    assert rel < 1e-3, rel
    assert abs(float(st.grad) - want_s) <= 1e-3 * abs(want_s)
    # The forward is the engine's kernel: it matches the FP32 oracle frame.
    h2 = oracle.h2_inv_norm(strength, s)
    ref = oracle.nlm_frame([f for f in window], d, a, s, h2)
    assert np.abs(out.detach().cpu().numpy() - ref[..., 0]).max() < 2e-5


def test_sure_picks_a_strength_that_lowers_the_error():
    import torch

    from av_denoise_b200 import synth
    from av_denoise_b200.autograd import NlmWindow, sure

    d, a, s = 2, 5, 2
    sigma = 16.0 / 1023.0
    clip = synth.make_clip(128, 128, 1, depth=10, chroma="gray", sigma_luma=0.0, global_motion=0, sprites=0,
                           seed=4)
    clean = torch.from_numpy(clip[0][0].astype(np.float32) / 1023.0).cuda()
    gen = torch.Generator(device="cuda").manual_seed(0)
    noisy = torch.stack([clean + sigma * torch.randn(clean.shape, generator=gen, device="cuda")
                         for _ in range(2 * d + 1)])
    log_h = torch.tensor(float(np.log(12.0)), device="cuda", requires_grad=True)  # start well above
    opt = torch.optim.Adam([log_h], lr=0.05)

    def mse(h):
        with torch.no_grad():
            return float(((NlmWindow.apply(noisy, h, d, a, s) - clean) ** 2).mean())

    start_mse = mse(log_h.exp().detach())
    sures = []
    for _ in range(50):
        opt.zero_grad()
        loss = sure(noisy, log_h.exp(), sigma, d, a, s, probes=16, generator=gen)
        loss.backward()
        opt.step()
        sures.append(float(loss.detach()))
    end_mse = mse(log_h.exp().detach())
    print("strength", float(log_h.exp()), "mse", start_mse, "->", end_mse, "sure", sures[0], "->", sures[-1])
    assert sures[-1] < sures[0]
    assert end_mse < start_mse
