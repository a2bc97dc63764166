"""The parity bar at full size on the two NLMeans workloads: every sample of every frame through the
engine, against the FP32 oracle on the same seeded frames.

Bar: no sample more than 1 LSB from the oracle and at least 99.9% of all samples identical (raw,
ties included). The window kernel flags the samples whose float result lies near a change of code
and the exact finish recomputes them in the oracle's operation order, so the codes agree exactly.

- the 640x360 spatial workload: 8 luma frames (u8), frame k shifted by (k, k/2), sigma 10,
  d=0, a=7, s=3, strength 12 (h = 1.2 sigma / 255 in normalised units);
- the 1080p temporal workload: 8 frames of the seeded 1920x1080 4:2:0 u8 clip (pan in [-4, 4],
  three 200x200 sprites, sigma 8 luma / 5 chroma), a luma engine (d=2, a=5, s=2, strength 8) and a
  chroma engine (d=0, a=5, s=2, strength 5), as a reference caller runs them.
"""

import numpy as np
import pytest

from conftest import avd
from gpu_util import Parity, Runner, oracle_pass

pytestmark = pytest.mark.gpu


def fast(d, a, s, strength):
    mode = avd.DenoisingMode.temporal(d) if d else avd.DenoisingMode.spacial()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s, strength=strength)
    return avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=tuning, mode=mode))


def _check(par: Parity):
    st = par.stats()
    print(st)
    assert st["max_lsb"] <= 1, st
    assert st["identical"] >= 0.999, st
    return st


def test_spatial_640x360_full_frames(oracle):
    from av_denoise_b200 import synth

    frames = synth.spatial_clip(seed=0, frames=8)
    fmt = avd.SampleFormat.u8()
    spec = avd.EngineSpec.nlmeans(fast(0, 7, 3, 12.0), None,
                                  avd.Geometry(640, 360, avd.ChromaLayout.GRAY, fmt, fmt))
    got = Runner(spec).run(frames)
    want = oracle_pass(oracle, frames, fmt, 0, 7, 3, 12.0)
    assert len(got) == len(want) == 8
    par = Parity()
    for g, w in zip(got, want):
        par.add(g[0], w[0], None, 255.0)
    _check(par)


def test_temporal_1080p_full_frames(oracle):
    from av_denoise_b200 import synth

    frames = synth.temporal_1080p_clip(seed=1000, frames=8)
    fmt = avd.SampleFormat.u8()
    geo = avd.Geometry(1920, 1080, avd.ChromaLayout.YUV420, fmt, fmt)
    luma = Runner(avd.EngineSpec.nlmeans(fast(2, 5, 2, 8.0), None, geo)).run(frames)
    chroma = Runner(avd.EngineSpec.nlmeans(None, fast(0, 5, 2, 5.0), geo)).run(frames)
    want_y = oracle_pass(oracle, [[f[0]] for f in frames], fmt, 2, 5, 2, 8.0)
    want_uv = oracle_pass(oracle, [[f[1], f[2]] for f in frames], fmt, 0, 5, 2, 5.0, chroma=True)
    par_y, par_uv = Parity(), Parity()
    for k in range(8):
        par_y.add(luma[k][0], want_y[k][0], None, 255.0)
        for c in range(2):
            par_uv.add(chroma[k][1 + c], want_uv[k][c], None, 255.0)
        # each engine passes the other plane group through untouched
        assert np.array_equal(luma[k][1], frames[k][1]) and np.array_equal(chroma[k][0], frames[k][0])
    _check(par_y)
    _check(par_uv)
