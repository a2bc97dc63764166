"""The block-matching motion search on the GPU through the C ABI against the CPU oracle: pyramid
values, vectors and confidences bit for bit (every SAD is a sequential f32 sum in the reference's
order, and the confidence one correctly rounded division)."""

import ctypes as C

import numpy as np
import pytest

from motion_cases import moving_window

pytestmark = pytest.mark.gpu

CASES = [
    # width, height, frames, levels, blksize, overlap, radius, channels, confidence
    (160, 96, 5, 2, 16, 8, 4, 1, True),
    (123, 77, 3, 3, 16, 8, 6, 2, True),
    (64, 48, 3, 1, 8, 4, 2, 1, False),
    (200, 120, 5, 2, 32, 16, 8, 1, True),
    (96, 64, 5, 1, 16, 8, 0, 1, True),
    (33, 17, 3, 2, 8, 0, 3, 1, True),
]


def gpu_search(lib, ring, w, h, frames, levels, blksize, overlap, radius, channels, confidence, centre, slots,
               sad_floor, thsad):
    import torch

    from av_denoise_b200 import _abi

    dev = torch.from_numpy(ring.reshape(-1)).cuda()
    pyr = torch.zeros(lib.avd_motion_pyramid_floats(w, h, frames, levels), dtype=torch.float32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for s in range(frames):
        assert lib.avd_motion_pyramid_build(dev.data_ptr(), channels, w, h, frames, s, levels, pyr.data_ptr(), s,
                                            stream) == 0
    step = blksize - overlap
    bx, by = max(-(-w // step), 1), max(-(-h // step), 1)
    n = len(slots)
    slots_t = torch.tensor(np.asarray(slots, np.int32), device="cuda")
    mv = torch.zeros(n * bx * by * 2, dtype=torch.int32, device="cuda")
    conf = torch.zeros(n * bx * by, dtype=torch.float32, device="cuda")
    noise = torch.tensor([sad_floor], dtype=torch.float32, device="cuda")
    p = _abi.AvdMotionPass()
    p.pyramid, p.neighbour_slots, p.mv_field = pyr.data_ptr(), slots_t.data_ptr(), mv.data_ptr()
    p.confidence = conf.data_ptr() if confidence else 0
    p.noise = noise.data_ptr()
    p.width, p.height, p.frame_count, p.centre_slot, p.neighbours = w, h, frames, centre, n
    p.blksize, p.overlap, p.search_radius, p.levels = blksize, overlap, radius, levels
    p.mv_stride, p.conf_stride, p.sad_floor_word, p.thsad = bx * by * 2, bx * by, 0, thsad
    st = lib.avd_motion_search(C.byref(p), stream)
    assert st == 0, lib.avd_last_error().decode()
    torch.cuda.synchronize()
    return pyr.cpu().numpy(), mv.cpu().numpy().reshape(n, bx * by, 2), conf.cpu().numpy().reshape(n, bx * by)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[:7])))
def test_motion_search_matches_oracle_bit_for_bit(lib, oracle, case):
    w, h, frames, levels, blksize, overlap, radius, channels, confidence = case
    ring = moving_window(w, h, frames, seed=w * 7 + h, channels=channels)
    centre = frames // 2
    slots = [s for s in range(frames) if s != centre][::-1]
    floor = oracle.sad_noise_floor(blksize, 0.02)
    th = oracle.thsad(blksize, 1.0)
    pyr, mv, conf = gpu_search(lib, ring, w, h, frames, levels, blksize, overlap, radius, channels, confidence,
                               centre, slots, floor, th)
    o_pyr = oracle.motion_pyramid(ring, channels, w, h, levels)
    assert np.array_equal(pyr.view(np.uint32), o_pyr.view(np.uint32))
    o_mv, o_conf = oracle.motion_search(o_pyr, w, h, frames, centre, slots, blksize=blksize, overlap=overlap,
                                        search_radius=radius, levels=levels, confidence=confidence,
                                        sad_floor=floor, thsad=th)
    assert np.array_equal(mv, o_mv), np.argwhere(mv != o_mv)[:5]
    if confidence:
        assert np.array_equal(conf.view(np.uint32), o_conf.view(np.uint32))
        assert 0.0 <= conf.min() and conf.max() <= 1.0
