"""The NL4D collaborative-filter pass on the GPU through the C ABI (`avd_collab_pass`), against
the reference's recorded digests (collab/tests/fused/recorded.rs) with the reference's own
tolerances, and against the CPU oracle's accumulators."""

import ctypes as C

import numpy as np
import pytest

from collab_cases import GOLDEN, assert_matches_recorded, digest, recorded_cases
from conftest import avd

pytestmark = pytest.mark.gpu

CASES = recorded_cases()


def run_gpu(case: dict):
    import torch

    from av_denoise_b200 import _abi

    lib = avd.load()
    w, h, ch = case["width"], case["height"], case["channels"]
    ring = np.ascontiguousarray(case["ring"], np.float32)
    frames = ring.size // (w * h * ch)
    radius = case.get("radius", 0)
    sr = case.get("spatial_radius", 4)
    rho = case.get("rho", 0.0)
    profile = np.empty(8, np.float32)
    lib.avd_dct_noise_profile(rho, profile.ctypes.data_as(C.POINTER(C.c_float)))
    kaiser = np.empty(8, np.float32)
    lib.avd_kaiser_window(case.get("kaiser_beta", 0.0), kaiser.ctypes.data_as(C.POINTER(C.c_float)))
    sigma = float(case.get("sigma", (0.02,))[0])
    f = np.float32
    g = f(profile.max())
    ws = ((f(sigma) * f(sigma)) * g) * g
    ws = ws if np.isfinite(ws) and ws > f(1e-12) else f(1e-12)
    noise = np.array([sigma, sigma, ws, 0.0], np.float32)
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).cuda()  # noqa: E731
    dev = {
        "ring": t(ring, np.float32),
        "mv": t(case.get("mv_field", np.zeros(2, np.int32)), np.int32),
        "conf": t(case.get("confidence", np.ones(1, np.float32)), np.float32),
        "slots": t(np.asarray(case.get("neighbour_slots", np.zeros(1, np.uint32)), np.uint32).view(np.int32),
                   np.int32),
        "noise": t(noise, np.float32),
        "curve": t(np.zeros(16, np.float32), np.float32),
        "prof": t(profile, np.float32),
        "kaiser": t(kaiser, np.float32),
        "accum": torch.zeros(w * h * ch * frames, dtype=torch.int32, device="cuda"),
        "wsum": torch.zeros(w * h * frames, dtype=torch.int32, device="cuda"),
        "members": torch.zeros(lib.avd_collab_member_bytes(w, h) // 4, dtype=torch.int32, device="cuda"),
        "gw": torch.zeros(((w - 8 + 3) // 4 + 1) * ((h - 8 + 3) // 4 + 1), dtype=torch.float32, device="cuda"),
    }
    p = _abi.AvdCollabPass()
    p.ring, p.mv_field, p.confidence = dev["ring"].data_ptr(), dev["mv"].data_ptr(), dev["conf"].data_ptr()
    p.neighbour_slots, p.noise, p.noise_curve = dev["slots"].data_ptr(), dev["noise"].data_ptr(), dev["curve"].data_ptr()
    p.dct_profile, p.kaiser = dev["prof"].data_ptr(), dev["kaiser"].data_ptr()
    p.accum, p.wsum, p.group_weight = dev["accum"].data_ptr(), dev["wsum"].data_ptr(), dev["gw"].data_ptr()
    p.members = dev["members"].data_ptr()
    p.width, p.height, p.channels, p.centre_slot = w, h, ch, case.get("centre_slot", 0)
    p.sigma_word, p.weight_scale_word, p.curve_valid_word = 0, 2, 3
    p.radius, p.refine, p.spatial_radius, p.k_max = radius, case.get("refine", 0), sr, case.get("k_max", 8)
    p.mv_stride, p.conf_stride = case.get("mv_stride", 2), case.get("conf_stride", 1)
    p.blk_step, p.blksize = 8, 16
    p.blocks_x, p.blocks_y = case.get("blocks_x", 1), case.get("blocks_y", 1)
    p.pooled = int(case.get("pooled") is not None)
    p.c_min, p.lambda_ht = case.get("c_min", 0.0), case.get("lambda_ht", 5.3)
    p.accum_scale = lib.avd_cross_frame_accum_scale(sr, radius)
    p.pool_ratio = case.get("pooled") or 0.0
    st = lib.avd_collab_pass(C.byref(p), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    return dev["accum"].cpu().numpy(), dev["wsum"].cpu().numpy(), dev["gw"].cpu().numpy()


@pytest.mark.parametrize("label", list(CASES))
def test_gpu_matches_recorded_digest(oracle, label):
    case = CASES[label]
    accum, wsum, gw = run_gpu(case)
    assert_matches_recorded(label, digest(accum, wsum, gw), GOLDEN[label])
    # Against the oracle: the same pixels covered, and the accumulated pixels agree closely.
    kw = dict(case)
    o_acc, o_ws, o_gw = oracle.collab_fused(kw.pop("ring"), kw.pop("width"), kw.pop("height"), kw.pop("channels"),
                                            **kw)
    # Against the oracle: the kernels round every multiply and add as the restatement does and
    # aggregate in integers, so the accumulators and group weights are identical.
    assert np.array_equal(accum, o_acc)
    assert np.array_equal(wsum, o_ws)
    assert np.array_equal(gw.view(np.uint32), o_gw.view(np.uint32))


@pytest.mark.parametrize("w,h,radius,sr,seed", [(96, 64, 2, 4, 1), (61, 45, 1, 9, 2), (80, 56, 2, 6, 3),
                                                (96, 64, 0, 4, 4), (72, 40, 3, 5, 5)])
def test_gpu_matches_oracle_on_random_passes(oracle, w, h, radius, sr, seed):
    """Random textured frames, motion fields and confidences: the accumulators, weights and group
    weights equal the oracle's exactly."""
    rng = np.random.default_rng(seed)
    frames = 2 * radius + 1
    y, x = np.mgrid[0:h * frames, 0:w].astype(np.float32)
    ring = np.clip(0.5 + 0.2 * np.sin(x * 0.3 + y * 0.11) + rng.normal(0, 0.05, (h * frames, w)), 0, 1)
    case = dict(ring=ring.astype(np.float32).reshape(-1), width=w, height=h, channels=1, centre_slot=radius,
                radius=radius, c_min=0.3, refine=2, spatial_radius=sr, k_max=8, sigma=(0.03,), lambda_ht=3.0,
                rho=0.0, kaiser_beta=2.0)
    if radius:
        bx, by = -(-w // 8), -(-h // 8)
        case.update(mv_field=rng.integers(-6, 7, 2 * radius * bx * by * 2).astype(np.int32),
                    confidence=rng.uniform(0, 1, 2 * radius * bx * by).astype(np.float32),
                    neighbour_slots=np.array([s for s in range(frames) if s != radius], np.uint32),
                    mv_stride=bx * by * 2, conf_stride=bx * by, blocks_x=bx, blocks_y=by)
    case["pooled"] = 2.42 / 4.158 if seed % 2 else None
    accum, wsum, gw = run_gpu(case)
    kw = dict(case)
    o_acc, o_ws, o_gw = oracle.collab_fused(kw.pop("ring"), kw.pop("width"), kw.pop("height"), kw.pop("channels"),
                                            **kw)
    assert np.array_equal(wsum, o_ws)
    assert np.array_equal(accum, o_acc)
    assert np.array_equal(gw.view(np.uint32), o_gw.view(np.uint32))
