"""The launch tuner on the GPU: an engine tuning its window kernel (Auto, with a store) gives the
same samples as the baseline (Off); its choice lands in the store as one line per shape with every
variant's time, a later engine of that shape reuses it without timing again, and Cached mode reads
it from the file."""

import json

import pytest

from conftest import avd
from gpu_util import Runner

pytestmark = pytest.mark.gpu


def spec(w, h, d=2, a=5, s=2):
    fmt = avd.SampleFormat.u8()
    tuning = avd.NlmTuning(search_radius=a, patch_radius=s, strength=8.0)
    alg = avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=tuning, mode=avd.DenoisingMode.temporal(d)))
    return avd.EngineSpec.nlmeans(alg, alg, avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt))


def test_tuned_engine_matches_the_baseline_and_stores_its_choice(lib, tmp_path):
    from av_denoise_b200 import synth

    lib.avd_tune_forget()
    w, h = 256, 144
    frames = synth.make_clip(w, h, 6, chroma="420", sigma_luma=8.0, sigma_chroma=5.0, global_motion=2, seed=4)
    off = Runner(spec(w, h), tuning=avd.TuningConfig(mode="off")).run(frames)
    store = str(tmp_path)
    tuned = Runner(spec(w, h), tuning=avd.TuningConfig(mode="auto", store=store)).run(frames)
    for a, b in zip(off, tuned):
        for pa, pb in zip(a, b):
            assert (pa == pb).all()
    with open(store + "/av-denoise-b200-tune.jsonl") as f:
        rows = [json.loads(line) for line in f if line.strip()]
    keys = sorted(r["key"] for r in rows)
    assert len(rows) == 2 and any("c1 s2 a5 d2" in k for k in keys) and any("c2 s2 a5 d2" in k for k in keys)
    assert all(len(r["ms"]) == 3 and all(t > 0 for t in r["ms"]) and r["variant"] in (0, 1, 2) for r in rows)
    # The same shape again: remembered, no new timing.
    Runner(spec(w, h), tuning=avd.TuningConfig(mode="auto", store=store)).run(frames[:3])
    with open(store + "/av-denoise-b200-tune.jsonl") as f:
        assert len([line for line in f if line.strip()]) == 2
    lib.avd_tune_forget()
    cached = Runner(spec(w, h), tuning=avd.TuningConfig(mode="cached", store=store)).run(frames)
    for a, b in zip(off, cached):
        for pa, pb in zip(a, b):
            assert (pa == pb).all()
    lib.avd_tune_forget()
