"""The VapourSynth filter's frame pump on the GPU (av-denoise-vs/src/filter.rs over the host
denoiser): whatever order VapourSynth asks for output frames in (in order, a shuffled burst, a seek,
backwards, from several threads), every output equals the same clip streamed straight through the
host denoiser, for repeat-edge NLMeans and shifted-edge NL4D. Source frames arrive with padded row
strides, as VapourSynth lays them out."""

import threading

import numpy as np
import pytest

from conftest import avd
from av_denoise_b200 import vs_filter as vf

pytestmark = pytest.mark.gpu


class Source:
    """A 4:2:0 u8 clip served as strided planes (stride = width rounded up to 64 + 32 bytes)."""

    def __init__(self, frames):
        self.frames = frames
        self.num_frames = len(frames)
        self.height, self.width = frames[0][0].shape
        self.bytes_per_sample = 1
        self.fetched = 0

    def plane_dims(self, i):
        h, w = self.frames[0][i].shape
        return w, h

    def get_frame(self, index):
        self.fetched += 1
        out = []
        for p in self.frames[index]:
            h, w = p.shape
            stride = (w + 63) // 64 * 64 + 32
            buf = np.full((h, stride), 0xAA, np.uint8)
            buf[:, :w] = p
            out.append((buf.tobytes(), stride))
        return out


def straight(spec, frames):
    with avd.HostDenoiser(spec) as den:
        outs = []
        for f in frames:
            planes = [np.ascontiguousarray(p).tobytes() for p in f]
            try:
                den.push(planes)
            except avd.QueueFull:
                outs.append([bytes(p) for p in den.recv()])
                den.push(planes)
        den.flush(lambda planes: outs.append([bytes(p) for p in planes]))
    return outs


def specs(w, h):
    fmt = avd.SampleFormat.u8()
    geo = avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt)
    tuning = avd.NlmTuning(search_radius=3, patch_radius=2, strength=8.0)
    alg = avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=tuning, mode=avd.DenoisingMode.temporal(2)))
    o = avd.Nl4dOptions(sigma=8.0 / 255, temporal_radius=1, spatial_radius=4,
                        motion=avd.MotionSearch(estimation=avd.MotionEstimation.DIRECT))
    return {"nlm": avd.EngineSpec.nlmeans(alg, alg, geo), "nl4d": avd.EngineSpec.nl4d(o, o, geo)}


ORDERS = {
    "in_order": lambda n: list(range(n)),
    "shuffled": lambda n: [9, 0, 13, 4, 5, 6, 1, 12, 2, 11, 3, 10, 7, 8, 15, 14] + list(range(16, n)),
    "seek": lambda n: list(range(20, n)) + list(range(0, 20)),
    "backwards": lambda n: list(range(n - 1, -1, -1)),
}


@pytest.mark.parametrize("kind", ["nlm", "nl4d"])
@pytest.mark.parametrize("order", list(ORDERS))
def test_every_request_order_matches_the_straight_stream(kind, order):
    from av_denoise_b200 import synth

    w, h, n = 96, 64, 30
    frames = synth.make_clip(w, h, n, chroma="420", sigma_luma=8.0, sigma_chroma=5.0, global_motion=2, seed=n)
    spec = specs(w, h)[kind]
    want = straight(spec, frames)
    src = Source(frames)
    flt = vf.Denoise(src, spec, threads=4)
    try:
        for k in ORDERS[order](n):
            flt.get_frame_initial(k)
            got = flt.get_frame(k)
            assert got == want[k], (kind, order, k)
    finally:
        flt.close()


def test_requests_from_several_threads():
    from av_denoise_b200 import synth

    w, h, n = 96, 64, 24
    frames = synth.make_clip(w, h, n, chroma="420", sigma_luma=8.0, sigma_chroma=5.0, global_motion=2, seed=7)
    spec = specs(w, h)["nlm"]
    want = straight(spec, frames)
    flt = vf.Denoise(Source(frames), spec, threads=4)
    got, errors = {}, []

    def worker(start):
        try:
            for k in range(start, n, 4):
                flt.get_frame_initial(k)
                got[k] = flt.get_frame(k)
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(s,)) for s in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    flt.close()
    assert not errors
    assert all(got[k] == want[k] for k in range(n))


def test_unpacked_output_keeps_the_destination_padding():
    from av_denoise_b200 import synth

    w, h = 64, 48
    frames = synth.make_clip(w, h, 6, chroma="420", sigma_luma=8.0, sigma_chroma=5.0, seed=3)
    flt = vf.Denoise(Source(frames), specs(w, h)["nlm"], threads=2)
    flt.get_frame_initial(2)
    planes = flt.get_frame(2)
    flt.close()
    stride = 96
    dst = bytearray([0x55] * (stride * h))
    vf.unpack_plane_into(dst, stride, w, h, planes[0])
    arr = np.frombuffer(bytes(dst), np.uint8).reshape(h, stride)
    assert (arr[:, w:] == 0x55).all()
    assert arr[:, :w].tobytes() == planes[0]
