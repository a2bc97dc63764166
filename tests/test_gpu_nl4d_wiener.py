"""The NL4D Wiener stage and the collab pass's adjoint on the GPU, extensions with no counterpart in
the reference: the Wiener pass bit for bit against the f32 restatement, the adjoint
(`avd_collab_adjoint`) against the f64 restatement's adjoint (which the CPU tests check by central
differences), the torch.autograd harness over both, and the engine with the stage on against the
oracle's stream."""

import ctypes as C

import numpy as np
import pytest

from conftest import avd
from test_gpu_nl4d import check, clip, opts
from test_oracle_collab_adjoint import CASES, adjoint_case, f64

pytestmark = pytest.mark.gpu


def on_gpu(c):
    """The case's window and noise levels as CUDA tensors, and the harness's pass settings."""
    import torch

    from av_denoise_b200.autograd import Nl4dPassConfig

    k = c["case"]
    frames = 2 * k["radius"] + 1
    window = torch.from_numpy(c["ring"].reshape(frames, c["h"], c["w"], c["channels"]).copy()).cuda()
    sigma = torch.tensor(np.asarray(k["sigma"], np.float32), device="cuda")
    mv = torch.from_numpy(k["mv_field"]).cuda() if "mv_field" in k else None
    conf = torch.from_numpy(k["confidence"]).cuda() if "confidence" in k else None
    cfg = Nl4dPassConfig(radius=k["radius"], spatial_radius=k["spatial_radius"], refine=k["refine"],
                         lambda_ht=k["lambda_ht"], pool_ratio=k["pooled"], kaiser_beta=k["kaiser_beta"],
                         c_min=k["c_min"], wiener=k["wiener"], mv_field=mv, confidence=conf)
    return window, sigma, cfg


@pytest.mark.parametrize("seed,channels,radius,pooled,wiener", CASES)
def test_pass_matches_the_restatement(oracle, seed, channels, radius, pooled, wiener):
    """Hard, pooled and Wiener passes of 1 and 2 channels: the member words, accumulators and group
    weights equal the f32 restatement's bit for bit."""
    import torch

    from av_denoise_b200.autograd import _Nl4dState

    c = adjoint_case(seed, channels, radius, pooled, wiener)
    window, sigma, cfg = on_gpu(c)
    st = _Nl4dState(window, sigma, cfg)
    st.run()
    torch.cuda.synchronize()
    assert np.array_equal(st.members.cpu().numpy().view(np.uint32), c["record"]["members"])
    assert np.array_equal(st.accum.cpu().numpy(), c["accum"])
    assert np.array_equal(st.wsum.cpu().numpy(), c["wsum"])
    assert np.array_equal(st.group_weight.cpu().numpy().view(np.uint32), c["gw"].view(np.uint32))


@pytest.mark.parametrize("seed,channels,radius,pooled,wiener", CASES)
def test_adjoint_matches_the_f64_adjoint(oracle, seed, channels, radius, pooled, wiener):
    """Random dL/dA and dL/dW: the kernel's dL/d(ring) is the f64 adjoint's within 1e-4 of its norm
    (and 1e-3 of its largest entry everywhere), dL/d(sigma_c) within 1e-3 relative."""
    import torch

    from av_denoise_b200 import _abi
    from av_denoise_b200.autograd import _Nl4dState

    lib = avd.load()
    c = adjoint_case(seed, channels, radius, pooled, wiener)
    window, sigma, cfg = on_gpu(c)
    st = _Nl4dState(window, sigma, cfg)
    st.run()
    rng = np.random.default_rng(200 + seed)
    ga = rng.normal(0, 1, c["accum"].shape).astype(np.float32)
    gw = rng.normal(0, 1, c["wsum"].shape).astype(np.float32)
    grad_ring = torch.zeros_like(window)
    grad_refs = torch.empty(st.refs * channels, dtype=torch.float32, device="cuda")
    ga_d, gw_d = torch.from_numpy(ga).cuda(), torch.from_numpy(gw).cuda()
    adj = _abi.AvdCollabAdjoint(ga_d.data_ptr(), gw_d.data_ptr(), grad_ring.data_ptr(), grad_refs.data_ptr())
    code = lib.avd_collab_adjoint(C.byref(st.p), C.byref(adj), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert code == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    want_ring, want_sigma = f64(c, grads=(ga.astype(np.float64), gw.astype(np.float64)))
    got_ring = grad_ring.cpu().numpy().reshape(-1).astype(np.float64)
    err = got_ring - want_ring
    assert np.linalg.norm(err) <= 1e-4 * np.linalg.norm(want_ring)
    assert np.abs(err).max() <= 1e-3 * np.abs(want_ring).max()
    got_sigma = grad_refs.view(st.refs, channels).sum(0).cpu().numpy().astype(np.float64)
    for ch in range(channels):
        assert abs(got_sigma[ch] - want_sigma[ch]) <= 1e-3 * max(abs(want_sigma[ch]), 1.0), (ch, got_sigma, want_sigma)


@pytest.mark.parametrize("seed,channels,radius,pooled,wiener", [CASES[1], CASES[3], CASES[4], CASES[2]])
def test_autograd_harness(oracle, seed, channels, radius, pooled, wiener):
    """Nl4dPass: the forward is the pass's normalised centre frame (the restatement's accum x 5 /
    wsum, bit for bit), and backward is the adjoint of A / W at the pass's own accumulators: the
    gradients of <G, out> equal the f64 adjoint fed the same dL/dA = G / W and
    dL/dW = -<G, out> / W within 1e-4 of the window gradient's norm and 1e-3 of sigma's."""
    import torch

    from av_denoise_b200.autograd import Nl4dPass

    c = adjoint_case(seed, channels, radius, pooled, wiener)
    window, sigma, cfg = on_gpu(c)
    window.requires_grad_(True)
    sigma.requires_grad_(True)
    out = Nl4dPass.apply(window, sigma, cfg)
    frames, h, w, ch = window.shape
    acc = c["accum"].reshape(frames, h, w, ch)[radius].astype(np.float64)
    ws = c["wsum"].reshape(frames, h, w)[radius].astype(np.float64)
    want_out = (acc * 5.0 / ws[..., None]).astype(np.float32)
    assert np.array_equal(out.detach().cpu().numpy(), want_out)
    g = np.random.default_rng(7).normal(0, 1, out.shape).astype(np.float32)
    (out * torch.from_numpy(g).cuda()).sum().backward()
    # The accumulators in real units, as the harness reads them.
    scale = oracle.cross_frame_accum_scale(cfg.spatial_radius, radius)
    w_real = ws / (5.0 * scale)
    out_real = (acc / scale) / w_real[..., None]
    ga = np.zeros((frames, h, w, ch))
    gw = np.zeros((frames, h, w))
    ga[radius] = g / w_real[..., None]
    gw[radius] = -(g * out_real).sum(-1) / w_real
    want_ring, want_sigma = f64(c, grads=(ga.reshape(-1), gw.reshape(-1)))
    got = window.grad.cpu().numpy().reshape(-1)
    assert np.linalg.norm(got - want_ring) <= 1e-4 * np.linalg.norm(want_ring)
    got_sigma = sigma.grad.cpu().numpy()
    for k in range(ch):
        assert abs(got_sigma[k] - want_sigma[k]) <= 1e-3 * max(abs(want_sigma[k]), 1e-2), (k, got_sigma, want_sigma)


@pytest.mark.parametrize("pooled", [False, True])
def test_engine_wiener_matches_oracle(oracle, pooled):
    """The NL4D engine with the Wiener stage on, luma, Direct motion: every output sample equals the
    oracle stream's."""
    w, h, n, d, sigma = 80, 56, 6, 1, 12.0 / 255
    fmt = avd.SampleFormat.u8()
    frames = clip(w, h, n, seed=31)
    kw = dict(spatial_radius=6, pooled_threshold=pooled, wiener=True)
    if not pooled:
        kw.update(lambda_ht=2.7)
    spec = avd.EngineSpec.nl4d(opts(d, sigma, **kw), None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt))
    from gpu_util import Runner

    got = Runner(spec).run(frames)
    check(oracle, [[g[0]] for g in got], [[f[0]] for f in frames], fmt, d, sigma, **kw)
