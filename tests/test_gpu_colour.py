"""The colour grain gain kernels on the GPU through the C ABI, bit for bit against the oracle: the
block means of both grids at every sample format and subsampling, the cell sums of luma and chroma
passes, the window's sums, both fits with the gains, and the table lookup."""

import ctypes as C

import numpy as np
import pytest

import colour_cases as cc
from conftest import avd

pytestmark = pytest.mark.gpu


def stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1).copy()).cuda()


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _pack(codes, kind):
    codes = np.asarray(codes).reshape(-1)
    if kind == "f32":
        return np.ascontiguousarray(codes.astype(np.float32)).view(np.uint32)
    per, dt = (4, np.uint8) if kind == "u8" else (2, np.uint16)
    pad = (-len(codes)) % per
    return np.concatenate([codes.astype(dt), np.zeros(pad, dt)]).view(np.uint32)


@pytest.mark.parametrize("layout", ["420", "422", "444"])
@pytest.mark.parametrize("fmt", ["u8", "u10", "u16", "f32"])
@pytest.mark.parametrize("w,h", [(64, 48), (77, 45)])
def test_block_means_match_oracle(lib, oracle, layout, fmt, w, h):
    import torch

    sx, sy = {"420": (1, 1), "422": (1, 0), "444": (0, 0)}[layout]
    chroma = {"420": avd.ChromaLayout.YUV420, "422": avd.ChromaLayout.YUV422, "444": avd.ChromaLayout.YUV444}[layout]
    cw, ch = -(-w // (1 << sx)), -(-h // (1 << sy))
    rng = np.random.default_rng(w + h + sx)
    if fmt == "f32":
        sf, kind, spw = avd.SampleFormat.f32(), "f32", 1
        y = rng.random((h, w), np.float32)
        u, v = rng.random((ch, cw), np.float32) - 0.5, rng.random((ch, cw), np.float32) - 0.5
        scale, bias = 255.0, 0.5
    else:
        depth = {"u8": 8, "u10": 10, "u16": 16}[fmt]
        sf = avd.SampleFormat.u8() if depth == 8 else avd.SampleFormat.u16(depth)
        kind, spw = ("u8", 4) if depth == 8 else ("u16", 2)
        top = (1 << depth) - 1
        y = rng.integers(0, top + 1, (h, w))
        u, v = rng.integers(0, top + 1, (ch, cw)), rng.integers(0, top + 1, (ch, cw))
        scale, bias = float(np.float32(1.0) / np.float32(1 << (depth - 8))), 0.0
    planes = [_pack(y, kind), _pack(u, kind), _pack(v, kind)]
    geo = avd.Geometry(w, h, chroma, sf, sf)
    nl = -(-w // 16) * -(-h // 16)
    nc = -(-cw // 16) * -(-ch // 16)
    lm = torch.full((nl * 3,), -9.0, device="cuda")
    cm = torch.full((nc * 3,), -9.0, device="cuda")
    d = [dev(p) for p in planes]
    assert lib.avd_colour_means(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), C.byref(geo._c()), lm.data_ptr(),
                                cm.data_ptr(), stream()) == 0, lib.avd_last_error().decode()
    want_l, want_c = oracle.colour_means(*planes, w, h, sx, sy, spw, fmt == "f32", scale, bias)
    assert np.array_equal(bits(host(lm)), bits(want_l.reshape(-1)))
    assert np.array_equal(bits(host(cm)), bits(want_c.reshape(-1)))


def gpu_cells(lib, records, means, w, h, channels, luma):
    import torch

    words = lib.avd_colour_records(channels, int(luma)) * 69
    out = torch.full((words,), 77, dtype=torch.int32, device="cuda")
    r, m = dev(np.asarray(records, np.float32)), dev(np.asarray(means, np.float32))
    assert lib.avd_colour_accumulate(r.data_ptr(), m.data_ptr(), w, h, channels, int(luma), 255.0, out.data_ptr(),
                                     stream()) == 0, lib.avd_last_error().decode()
    return host(out)


@pytest.mark.parametrize("channels,luma", [(1, True), (2, False)])
def test_cell_sums_match_oracle(lib, oracle, channels, luma):
    B = cc.ColourBlock
    blocks = [B(100.0, 0.0, 0.0, 2.0), B.coloured(100.0, 9.0, 0, 2.0), B.coloured(100.0, 9.0, 11, 1.5),
              B.coloured(130.0, 16.0, 3, 3.0), B.coloured(130.0, 25.0, 6, 2.5), B.coloured(60.0, 37.0, 8, 1.2),
              B.coloured(60.0, 80.0, 5, 4.0), B(200.0, 3.0, -4.0, 0.8), B.coloured(200.0, 13.0, 9, 1.0),
              B.coloured(25.0, 50.0, 2, 2.0), B.coloured(235.0, 7.0, 7, 2.2), B.coloured(150.0, 44.5, 10, 0.6),
              B(20.0, 0.0, 0.0, 2.0), B(100.0, 5.99, 0.0, 2.0), B(100.0, 0.0, 0.0, 0.04),
              B(100.0, 0.0, 0.0, 2.0, mean=3.0)]
    run = cc.CellRun(oracle, 64, 64, channels, luma)
    records, colour = run.inputs(blocks)
    got = gpu_cells(lib, records, colour, 64, 64, channels, luma)
    want = oracle.colour_accumulate(records, colour, 64, 64, channels, luma, 255.0)
    assert np.array_equal(got, want)


@pytest.fixture(scope="module")
def scenes():
    def luma_grain(luma, cb, cr):
        g = (1.2 + luma / 200.0) * (1.0 + max(cr - cb, 0.0) / 40.0)
        return (g, g)

    return {
        "luma": cc.random_scene(60_000, 11, luma_grain),
        "chroma": cc.random_scene(60_000, 23, lambda luma, cb, cr: (0.8 + 0.6 * (max(cb, 0.0) / 30.0) + luma / 400.0,
                                                                     0.6 + 0.9 * (abs(cr) / 40.0))),
        "planted": cc.cell_scene(220, 5, range(2, 14), cc.planted_factor),
        "thin": cc.cell_scene(5, 9, range(2, 14), cc.planted_factor),
    }


@pytest.mark.parametrize("scene,planes,luma,ratios,curve_valid", [
    ("luma", 1, True, cc.RISING_CURVE, True),
    ("luma", 1, True, cc.RISING_CURVE, False),
    ("chroma", 2, False, cc.FLAT_CURVE, False),
    ("planted", 1, True, cc.FLAT_CURVE, True),
    ("planted", 2, False, cc.FLAT_CURVE, False),
    ("thin", 1, True, cc.FLAT_CURVE, True),
])
def test_window_and_fit_match_oracle(lib, oracle, scenes, scene, planes, luma, ratios, curve_valid):
    import torch

    window, frames, ring = cc.fit_window(oracle, scenes[scene], planes, luma)
    # The cell sums of every frame and the window over them, on the GPU.
    w, h = cc.FRAME_WIDTH, (cc.FRAME_BLOCKS // 64) * 16
    cap, words = ring.shape
    gring = torch.zeros(cap * words, dtype=torch.int32, device="cuda")
    for f, (records, means) in enumerate(frames):
        r, m = dev(records), dev(means)
        slot = gring[f * words:(f + 1) * words]
        assert lib.avd_colour_accumulate(r.data_ptr(), m.data_ptr(), w, h, planes, int(luma), 255.0, slot.data_ptr(),
                                         stream()) == 0
    gwin = torch.full((words,), -1.0, device="cuda")
    assert lib.avd_colour_window(gring.data_ptr(), cap, 0, len(frames) - 1, words, gwin.data_ptr(), stream()) == 0
    assert np.array_equal(host(gring).reshape(cap, words), ring)
    assert np.array_equal(bits(host(gwin)), bits(window))
    # Both fits and the gains.
    derived = np.zeros(16, np.float32)
    derived[3] = 1.0 if curve_valid else 0.0
    dcurve, dder = dev(np.asarray(ratios, np.float32)), dev(derived)
    scratch = torch.full((lib.avd_colour_fit_scratch_floats(planes),), -3.0, device="cuda")
    table = torch.full((planes * 976,), -3.0, device="cuda")
    gains = torch.full((planes * 976,), -3.0, device="cuda")
    assert lib.avd_colour_fit(gwin.data_ptr(), planes, int(luma), dcurve.data_ptr(), dder.data_ptr(),
                              scratch.data_ptr(), table.data_ptr(), gains.data_ptr(), stream()) == 0, \
        lib.avd_last_error().decode()
    want_table, want_gains, _ = oracle.colour_fit(window, planes, luma, ratios, curve_valid)
    got_table, got_gains = host(table), host(gains)
    assert np.array_equal(bits(got_table), bits(want_table)), np.abs(got_table - want_table).max()
    assert np.array_equal(bits(got_gains), bits(want_gains)), np.abs(got_gains - want_gains).max()
    # The lookup at colours spread over the table and just past its edges.
    rng = np.random.default_rng(planes)
    q = np.stack([300 * rng.random(2048) - 20, 180 * rng.random(2048) - 90, 180 * rng.random(2048) - 90], 1)
    q = q.astype(np.float32)
    for p in range(planes):
        tab = dev(want_gains[p * 976:(p + 1) * 976])
        vals = torch.zeros(len(q), device="cuda")
        gn = torch.zeros(len(q), device="cuda")
        assert lib.avd_colour_lookup(tab.data_ptr(), dev(q).data_ptr(), len(q), vals.data_ptr(), gn.data_ptr(),
                                     stream()) == 0
        wv, wg = oracle.colour_lookup(want_gains[p * 976:(p + 1) * 976], q)
        assert np.array_equal(bits(host(vals)), bits(wv)) and np.array_equal(bits(host(gn)), bits(wg))
