"""Throughput of the NLMeans hot path on B200.

Workload (one step = the whole clip): 32 frames of 1920x1080 4:2:0 8-bit, luma NLMeans with
temporal radius 2, search radius 5, patch radius 2, strength 8 (h = 8/255); chroma NLMeans spatial,
search radius 5, patch radius 2, strength 5. The reference rejects one engine with mixed luma and
chroma window spans, so, as a reference caller must, two engines run side by side: one cleans
luma (chroma passed through), one cleans chroma (luma passed through).

  value : frames/s with the clip resident in HBM (push + emit through the engine API, device
          planes), L2 flushed between steps, timed with CUDA events on the engine stream.
  e2e   : frames/s through the same API from pinned host memory: every step copies each frame's
          planes host->device, denoises, and copies the result device->host, on two streams.
  --impl reference : the reference's CPU path is not runnable here (its CPU device is a software
          Vulkan renderer, and the Rust crate cannot be built), so that arm times the CPU
          restatement of the reference kernels (oracle/, all host threads) on a bounded crop.

Multi-GPU: clips are independent, so N ranks run N replicas with no data-path collective
(weak scaling); value = frames of all ranks / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import os
import tempfile
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

W, H, FRAMES = 1920, 1080, 32
LUMA = dict(d=2, a=5, s=2, strength=8.0)
CHROMA = dict(d=0, a=5, s=2, strength=5.0)
METRIC = "frames/s 1080p+4K NLMeans/NL4D on 1 B200, batched & plain, ≤1 LSB vs ref"


def n_off(d: int, a: int) -> int:
    side = 2 * a + 1
    return side * side - 1 + 2 * d * side * side


def read_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        d["source"] = "measured"
        return d
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0, "source": "fallback"}


def clocks_start(path: Path):
    cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "200", "-i", os.environ.get("LOCAL_RANK", "0")]
    try:
        return subprocess.Popen(cmd, stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def clocks_stop(proc, path: Path) -> dict:
    if proc is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    proc.terminate()
    proc.wait(timeout=5)
    sms, maxes, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in path.read_text().splitlines():
        parts = [x.strip() for x in line.split(",")]
        if len(parts) < 9:
            continue
        try:
            sms.append(float(parts[1]))
            maxes.append(float(parts[2]))
        except ValueError:
            continue
        for n, v in zip(names, parts[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxes) if maxes else None,
            "reasons": sorted(reasons), "samples": len(sms)}


def build_specs(avd):
    fmt = avd.SampleFormat.u8()
    geo = avd.Geometry(W, H, avd.ChromaLayout.YUV420, fmt, fmt)

    def alg(p):
        mode = avd.DenoisingMode.temporal(p["d"]) if p["d"] else avd.DenoisingMode.spacial()
        t = avd.NlmTuning(search_radius=p["a"], patch_radius=p["s"], strength=p["strength"])
        return avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=t, mode=mode))

    return avd.EngineSpec.nlmeans(alg(LUMA), None, geo), avd.EngineSpec.nlmeans(None, alg(CHROMA), geo)


def replica_seed(rank: int) -> int:
    """Each rank denoises its own clip (independent units, no data-path collective)."""
    return 1000 + rank


def replica_throughput(local_times: list[float], frames_per_rank: int, world: int, device: str = "cuda"):
    """Whole-job throughput of N replicas: every rank's timings are reduced to the max over ranks
    (the one collective, on timings only), and value = frames of all ranks / that time. Returns
    (max-over-ranks times, values)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(local_times, device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    times = [float(x) for x in t]
    return times, [frames_per_rank * world / x for x in times]


def plane_words(fmt, w, h):
    return fmt.plane_bytes(w * h) // 4


def _words_u8(np, codes):
    flat = codes.reshape(-1)
    return np.concatenate([flat, np.zeros((-flat.size) % 4, np.uint8)]).view(np.int32)


def oracle_frame(clip, k: int) -> tuple[list, float]:
    """The oracle's output planes (Y, U, V codes) of frame k of the workload and the seconds it took:
    the luma pass over the repeat-edge window of frame k, the chroma pass on frame k alone (FP32
    mirror, OpenMP on every host thread)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    oracle.build()
    n = len(clip)
    t0 = time.perf_counter()
    window = [oracle.ingest([clip[min(max(k + j, 0), n - 1)][0]], 0, 255.0) for j in range(-LUMA["d"], LUMA["d"] + 1)]
    y = oracle.nlm_frame(window, LUMA["d"], LUMA["a"], LUMA["s"], oracle.h2_inv_norm(LUMA["strength"], LUMA["s"]))
    uv = oracle.nlm_frame([oracle.ingest([clip[k][1], clip[k][2]], 0, 255.0)], 0, CHROMA["a"], CHROMA["s"],
                          oracle.h2_inv_norm(CHROMA["strength"], CHROMA["s"]))
    secs = time.perf_counter() - t0
    return oracle.egress(y, 0, 255.0) + oracle.egress(uv, 0, 255.0), secs


def run_gpu(args) -> None:
    import numpy as np
    import torch
    import torch.distributed as dist

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    clip = synth.temporal_1080p_clip(frames=FRAMES, seed=replica_seed(rank))
    spec_l, spec_c = build_specs(avd)
    fmt = spec_l.geometry.input
    dims = [spec_l.geometry.plane_dims(i) for i in range(3)]
    # The luma and chroma engines run on two streams: chroma's short launches fill the luma
    # launches' last wave.
    sl, sc = torch.cuda.Stream(), torch.cuda.Stream()
    eng_l = avd.build_engine(spec_l)
    eng_c = avd.build_engine(spec_c)
    eng_l.set_stream(sl.cuda_stream)
    eng_c.set_stream(sc.cuda_stream)

    dev_in = [[torch.from_numpy(_words_u8(np, p)).cuda() for p in f] for f in clip]
    out = [torch.zeros(plane_words(fmt, w, h), dtype=torch.int32, device="cuda") for (w, h) in dims]
    scratch = [torch.zeros(plane_words(fmt, w, h), dtype=torch.int32, device="cuda") for (w, h) in dims]
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def P(bufs):
        return [avd.DevicePlane.from_tensor(b, w, h) for b, (w, h) in zip(bufs, dims)]

    out_l = P([out[0], scratch[1], scratch[2]])
    out_c = P([scratch[0], out[1], out[2]])
    planes_in = [P(f) for f in dev_in]

    def step_device(capture: int = -1):
        """One pass of the clip through both engines; with `capture`, also that frame's planes."""
        got = {}
        emitted_l = emitted_c = 0

        def emit_l():
            nonlocal emitted_l
            eng_l.emit_into(out_l)
            if emitted_l == capture:
                with torch.cuda.stream(sl):
                    got["y"] = out[0].clone()
            emitted_l += 1

        def emit_c():
            nonlocal emitted_c
            eng_c.emit_into(out_c)
            if emitted_c == capture:
                with torch.cuda.stream(sc):
                    got["uv"] = (out[1].clone(), out[2].clone())
            emitted_c += 1

        for pl in planes_in:
            for _ in range(eng_l.push(pl)):
                emit_l()
            for _ in range(eng_c.push(pl)):
                emit_c()
        for _ in range(eng_l.finish()):
            emit_l()
        for _ in range(eng_c.finish()):
            emit_c()
        return emitted_l, got

    def timed(fn):
        e0, e1, ec = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(sl)
        sc.wait_event(e0)
        res = fn()
        ec.record(sc)
        sl.wait_event(ec)
        e1.record(sl)
        torch.cuda.synchronize()
        return res, e0.elapsed_time(e1) / 1e3

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()

    clock_path = Path(tempfile.gettempdir()) / f"avd_bench_clocks_{os.getpid()}_rank{rank}.csv"
    proc = clocks_start(clock_path)
    eng_l.sample_device_time(1)
    times = []
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        barrier()
        (n, _), t = timed(step_device)
        assert n == FRAMES
        times.append(t)
    wall = time.perf_counter() - wall0
    nlm_timing = eng_l.timing().luma  # window kernel + exact finish per luma frame
    eng_l.sample_device_time(0)
    # The chroma engine's frame, sampled on one more (untimed) step so the timed steps carry only
    # the luma engine's sampling events.
    eng_c.sample_device_time(1)
    step_device()
    torch.cuda.synchronize()
    ct = eng_c.timing()
    chroma_timing = ct.chroma if ct.chroma is not None else ct.luma  # the chroma engine's one pass
    eng_c.sample_device_time(0)

    # End to end: pinned host frames -> device -> engines -> device -> pinned host. Output frame k
    # gathers its chroma when the chroma engine emits it (at push k) and its luma when the luma engine
    # does (d pushes later); a 4-slot device ring holds it between.
    host_in = [[torch.from_numpy(_words_u8(np, p)).pin_memory() for p in f] for f in clip]
    host_out = [[torch.empty(plane_words(fmt, w, h), dtype=torch.int32).pin_memory() for (w, h) in dims]
                for _ in range(FRAMES)]
    stage = [[torch.empty(plane_words(fmt, w, h), dtype=torch.int32, device="cuda") for (w, h) in dims]
             for _ in range(2)]
    dout = [[torch.empty(plane_words(fmt, w, h), dtype=torch.int32, device="cuda") for (w, h) in dims]
            for _ in range(4)]
    dscr = [[torch.empty(plane_words(fmt, w, h), dtype=torch.int32, device="cuda") for (w, h) in dims]
            for _ in range(2)]
    copy = torch.cuda.Stream()
    h2d_bytes = sum(t.numel() * 4 for f in host_in for t in f)
    d2h_bytes = sum(t.numel() * 4 for f in host_out for t in f)

    def step_e2e():
        free_in = [[torch.cuda.Event() for _ in range(2)] for _ in range(2)]  # [slot][luma, chroma]
        free_out = [torch.cuda.Event() for _ in range(len(dout))]
        chroma_done = [torch.cuda.Event() for _ in range(len(dout))]
        for ev in free_out:
            ev.record(copy)
        for pair in free_in:
            pair[0].record(sl)
            pair[1].record(sc)
        luma_frame = chroma_frame = 0

        def emit_chroma():
            nonlocal chroma_frame
            o = chroma_frame % len(dout)
            sc.wait_event(free_out[o])
            eng_c.emit_into(P([dscr[1][0], dout[o][1], dout[o][2]]))
            chroma_done[o].record(sc)
            chroma_frame += 1

        def emit_luma():
            nonlocal luma_frame
            o = luma_frame % len(dout)
            eng_l.emit_into(P([dout[o][0], dscr[0][1], dscr[0][2]]))
            done = torch.cuda.Event()
            done.record(sl)
            copy.wait_event(done)
            copy.wait_event(chroma_done[o])
            with torch.cuda.stream(copy):
                for i in range(3):
                    host_out[luma_frame][i].copy_(dout[o][i], non_blocking=True)
            free_out[o].record(copy)
            luma_frame += 1

        for k, f in enumerate(host_in):
            s_ = k % 2
            copy.wait_event(free_in[s_][0])
            copy.wait_event(free_in[s_][1])
            with torch.cuda.stream(copy):
                for i in range(3):
                    stage[s_][i].copy_(f[i], non_blocking=True)
            ready = torch.cuda.Event()
            ready.record(copy)
            sl.wait_event(ready)
            sc.wait_event(ready)
            pl = P(stage[s_])
            for _ in range(eng_c.push(pl)):
                emit_chroma()
            free_in[s_][1].record(sc)
            for _ in range(eng_l.push(pl)):
                emit_luma()
            free_in[s_][0].record(sl)
        for _ in range(eng_c.finish()):
            emit_chroma()
        for _ in range(eng_l.finish()):
            emit_luma()
        return luma_frame

    for _ in range(max(3, args.warmup)):
        step_e2e()
    torch.cuda.synchronize()
    e2e_times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        n = step_e2e()
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
        assert n == FRAMES
    clocks = clocks_stop(proc, clock_path)

    # Output sanity: the e2e output of the last frame equals the resident run's.
    step_device()
    torch.cuda.synchronize()
    same = all(torch.equal(host_out[FRAMES - 1][i], out[i].cpu()) for i in range(3))

    # The dominant kernel alone: the luma window kernel with a float output (no exact finish), timed
    # by the engine's device timer over 16 frames of the same clip.
    f32 = avd.SampleFormat.f32()
    lspec = avd.EngineSpec.nlmeans(spec_l.luma, None, avd.Geometry(W, H, avd.ChromaLayout.GRAY, fmt, f32))
    eng_w = avd.build_engine(lspec)
    eng_w.set_stream(sl.cuda_stream)
    wbuf = torch.empty(W * H, dtype=torch.float32, device="cuda")
    wout = [avd.DevicePlane.from_tensor(wbuf, W, H)]
    for rep in range(2):
        eng_w.sample_device_time(1 if rep else 0)
        for f in planes_in[:16]:
            for _ in range(eng_w.push([f[0]])):
                eng_w.emit_into(wout)
        for _ in range(eng_w.finish()):
            eng_w.emit_into(wout)
    torch.cuda.synchronize()
    win_timing = eng_w.timing().luma
    eng_w.close()

    (t_step, t_e2e), (fps, fps_e2e) = replica_throughput(
        [sum(times) / len(times), sum(e2e_times) / len(e2e_times)], FRAMES, world)
    peaks = read_peaks()
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    luma_px = W * H
    ex2_per_launch = luma_px * n_off(LUMA["d"], LUMA["a"])
    t_window = win_timing.device_time / max(1, win_timing.frames)
    t_luma_frame = nlm_timing.device_time / max(1, nlm_timing.frames)
    achieved = ex2_per_launch / t_window / 1e9
    mufu_peak = sms * 16 * peaks["sm_max_mhz"] * 1e6 / 1e9
    hbm_bytes = luma_px * 4 * (2 * LUMA["d"] + 1) + luma_px * 4
    line = {
        "metric": METRIC,
        "value": round(fps, 2),
        "unit": "frames/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_step * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded gratings + rectangles + blurred texture, global pan and sprites, Gaussian noise)",
        "config": {"workload": "NLMeans 1920x1080 4:2:0 u8, 32 frames: luma d=2 a=5 s=2 strength 8; "
                               "chroma spatial a=5 s=2 strength 5 (a luma engine and a chroma engine on two "
                               "streams)", "frames_per_step": FRAMES,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "sfu", "kernel": "nlm_window_kernel<1,2,fast> (luma, 604 offsets/pixel)",
                     "achieved": round(achieved, 2), "peak": round(mufu_peak, 2), "unit": "Gex2/s",
                     "frac": round(achieved / mufu_peak, 4),
                     # dram__bytes_read.sum + dram__bytes_write.sum of one launch in an ncu capture of
                     # the same launch, not of this run.
                     "traffic": 41.52e6 + 0.151e6,
                     "traffic_source": "ncu capture: profiles/nlm_window_kernel_luma_1080p_d2a5s2.md",
                     "peak_note": f"MUFU ex2: {sms} SMs x 16/clk x sm_max_mhz {peaks['sm_max_mhz']} "
                                  f"({peaks['source']})",
                     "launch_ms": round(t_window * 1e3, 4),
                     "luma_frame_ms_with_exact_finish": round(t_luma_frame * 1e3, 4),
                     # pixels per luma frame the exact finish recomputed in the reference's order
                     "exact_samples_per_frame": round(nlm_timing.exact_samples / max(1, nlm_timing.frames), 1),
                     # the chroma engine's frame (window kernel + exact finish) on its own stream
                     "chroma_frame_ms_with_exact_finish": round(
                         chroma_timing.device_time / max(1, chroma_timing.frames) * 1e3, 4),
                     "chroma_exact_samples_per_frame": round(
                         chroma_timing.exact_samples / max(1, chroma_timing.frames), 1)},
        "roofline_hbm": {"bound": "hbm", "achieved": round(hbm_bytes / t_window / 1e9, 2),
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(hbm_bytes / t_window / 1e9 / peaks["hbm_gbs"], 5)},
        "e2e": {"value": round(fps_e2e, 2), "unit": "frames/s", "h2d_bytes_per_step": h2d_bytes,
                "d2h_bytes_per_step": d2h_bytes, "matches_resident_run": bool(same)},
        # per frame and engine: ingest, window, exact finish and egress
        "gpu_launches": 8 * FRAMES,
        "clocks": clocks,
        "wall_s_timed": round(wall, 3),
    }
    if rank == 0 and world == 1 and not args.no_nl4d:
        line["nl4d_4k"] = nl4d_4k_section(avd, torch, np, synth, pushes=args.nl4d_pushes)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # Parity of one full frame of the timed workload (outside the timed region) and the CPU
        # baseline: the oracle computes that frame once, timed.
        k = FRAMES // 2
        _, got = step_device(capture=k)
        torch.cuda.synchronize()
        gpu_planes = [got["y"], got["uv"][0], got["uv"][1]]
        want, secs = oracle_frame(clip, k)
        ident = total = max_lsb = 0
        for g, wn, (w, h) in zip(gpu_planes, want, dims):
            gv = g.cpu().numpy().view(np.uint8)[: w * h].reshape(h, w)
            d_ = np.abs(gv.astype(np.int64) - wn.astype(np.int64))
            ident += int((d_ == 0).sum())
            total += d_.size
            max_lsb = max(max_lsb, int(d_.max()))
        line["parity"] = {"frame": k, "samples": total, "identical": round(ident / total, 7), "max_lsb": max_lsb,
                          "against": "FP32 oracle (oracle/), one full 1920x1080 4:2:0 frame, luma and chroma"}
        line["cpu_baseline"] = {"value": round(1.0 / secs, 4), "unit": "frames/s", "cores": os.cpu_count(),
                                "kind": "port",
                                "sample": f"one full 1920x1080 4:2:0 frame (frame {k}: luma d=2 a=5 s=2 over its "
                                          "5-frame window + chroma a=5 s=2) through the FP32 oracle, OpenMP on "
                                          f"{os.cpu_count()} threads, {secs:.1f} s"}
    if rank == 0:
        print(json.dumps(line))
    eng_l.close()
    eng_c.close()
    if world > 1:
        dist.destroy_process_group()


def nl4d_4k_section(avd, torch, np, synth, pushes: int) -> dict:
    """The NL4D half of the metric on its 4K workload: 3840x2160 4:2:0 10-bit, 7-frame window (d=3,
    Auto resolves to Chained), spatial radius 16, hard threshold 2.7 (lambda_ht 2.7, scale 1, plain
    threshold), 12 sprites at up to 8 px/frame, noise 20 codes + 0.02 * value variance; sigma from
    the automatic noise estimate (motion-compensated look-ahead) on both plane groups, the luma noise
    map and the colour grain gains on (the reference's defaults), luma and chroma in one engine.
    Frames resident in HBM; device time per push with CUDA events, steady state after the window and
    look-ahead fill."""
    w, h, depth, d = 3840, 2160, 10, 3
    fmt = avd.SampleFormat.u16(depth)

    o = avd.Nl4dOptions(sigma=None, temporal_radius=d, spatial_radius=16, lambda_ht=2.7, lambda_ht_scale=1.0,
                        pooled_threshold=False)
    geo = avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt)
    engines = [avd.build_engine(avd.EngineSpec.nl4d(o, o, geo))]
    stream = torch.cuda.Stream()
    for eng in engines:
        eng.set_stream(stream.cuda_stream)
    clip = synth.make_clip(w, h, 12, depth=depth, chroma="420", sigma_luma=20.0 / 4.0, sigma_chroma=20.0 / 4.0,
                           sprites=12, sprite_speed=8, signal_dependent=0.02, seed=2000)
    dims = [geo.plane_dims(i) for i in range(3)]
    bufs = []
    for f in clip:
        planes = []
        for p in f:
            flat = p.reshape(-1).astype(np.uint16)
            planes.append(torch.from_numpy(np.concatenate([flat, np.zeros(flat.size % 2, np.uint16)]).view(np.int32)).cuda())
        bufs.append(planes)
    outs = [torch.zeros_like(b) for b in bufs[0]]

    def dp(ts):
        return [avd.DevicePlane.from_tensor(t, pw, ph) for t, (pw, ph) in zip(ts, dims)]

    times = []
    fill = 2 * d + 1 + 8
    for i in range(pushes):
        if i == fill:
            for eng in engines:
                eng.sample_device_time(1)  # events around every steady-state pass and its core launch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for eng in engines:
            for _ in range(eng.push(dp(bufs[i % len(bufs)]))):
                eng.emit_into(dp(outs))
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    timing = engines[0].timing()
    for eng in engines:
        eng.close()
    steady = times[fill:]
    ms = float(np.median(steady))

    # The group search's algorithmic FP32 operations per launch: every reference patch's clipped
    # centre window (33 x 33 inside the frame) and at least one 5 x 5 refine rectangle per volume
    # and neighbour frame, each candidate 64 squared differences per channel (sub, mul, add: the
    # oracle's unfused order) plus the group sum and the scale (8).
    def search_ops(pw, ph, c):
        def axis(n):
            top = n - 8
            return sum(min(min(i * 4, top) + 16, top) - max(min(i * 4, top) - 16, 0) + 1
                       for i in range((top + 3) // 4 + 1))
        refs = ((pw - 8 + 3) // 4 + 1) * ((ph - 8 + 3) // 4 + 1)
        per_candidate = 64 * c * 3 + 8
        return (axis(pw) * axis(ph) + refs * 2 * (2 * d) * 25) * per_candidate

    unfused_rate = 148 * 128 * 1.965e9  # FP32 lanes x the B200's top SM clock: one operation per lane per clock
    core = {}
    for name, t, (pw, ph), c in (("luma", timing.luma, dims[0], 1), ("chroma", timing.chroma, dims[1], 2)):
        if t is None or t.core_launches == 0:
            continue
        launch_s = t.core_time / t.core_launches
        ops = search_ops(pw, ph, c)
        core[name] = {"launch_ms": round(launch_s * 1e3, 3), "search_gops": round(ops / 1e9, 1),
                      "achieved_tops": round(ops / launch_s / 1e12, 2),
                      "frac_unfused_fp32": round(ops / launch_s / unfused_rate, 3)}
    return {"workload": "NL4D 3840x2160 4:2:0 10-bit luma+chroma, d=3 (Chained), spatial_radius 16, lambda_ht 2.7, "
                        "plain threshold; sigma automatic on both plane groups, noise map and colour gains on",
            "frames_per_s": round(1000.0 / ms, 2), "ms_per_frame": round(ms, 3), "pushes_timed": len(steady),
            "group_search": dict(core, note="CUDA events around each steady-state pass's group search + filter "
                                            "launch; operations counted for the search alone, so a lower bound")}


def run_reference(args) -> None:
    """The reference arm: the CPU restatement of the reference kernels (oracle/, FP32 mirror, OpenMP
    on every host thread) on the same workload. Each step is a bounded sample: frame k's central
    960x540 luma crop (d=2 over its 5-frame window) and 480x270 chroma crop, a quarter of a 1080p
    4:2:0 frame's pixels; frames/s is scaled to the full frame by that pixel ratio. Warm-up steps run
    the same sample untimed."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    import av_denoise_b200_loader

    av_denoise_b200_loader.load()
    from av_denoise_b200 import synth

    oracle.build()
    clip = synth.temporal_1080p_clip(frames=FRAMES, seed=1000)
    cw, ch = W // 2, H // 2
    x0, y0 = W // 4, H // 4
    h2_l = oracle.h2_inv_norm(LUMA["strength"], LUMA["s"])
    h2_c = oracle.h2_inv_norm(CHROMA["strength"], CHROMA["s"])

    def sample(k):
        t0 = time.perf_counter()
        win = [oracle.ingest([clip[min(max(k + j, 0), FRAMES - 1)][0][y0:y0 + ch, x0:x0 + cw]], 0, 255.0)
               for j in range(-LUMA["d"], LUMA["d"] + 1)]
        oracle.nlm_frame(win, LUMA["d"], LUMA["a"], LUMA["s"], h2_l)
        f = clip[k]
        uv = oracle.ingest([f[1][y0 // 2:y0 // 2 + ch // 2, x0 // 2:x0 // 2 + cw // 2],
                            f[2][y0 // 2:y0 // 2 + ch // 2, x0 // 2:x0 // 2 + cw // 2]], 0, 255.0)
        oracle.nlm_frame([uv], 0, CHROMA["a"], CHROMA["s"], h2_c)
        return time.perf_counter() - t0

    for i in range(args.warmup):
        sample(i % FRAMES)
    secs = [sample((args.warmup + i) % FRAMES) for i in range(args.steps)]
    per_step = statistics.mean(secs)
    fraction = (cw * ch) / (W * H)
    v = fraction / per_step
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(v, 4),
        "unit": "frames/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * per_step, 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "NLMeans 1920x1080 4:2:0 u8: luma d=2 a=5 s=2 strength 8; chroma spatial a=5 s=2 "
                               "strength 5", "frames_per_step": fraction,
                   "sample": f"per step: a central {cw}x{ch} luma crop (5-frame window) + {cw // 2}x{ch // 2} "
                             "chroma crop of one frame = 1/4 of a frame's pixels; frames/s scaled by 1/4"},
        "cpu_baseline": {"value": round(v, 4), "unit": "frames/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{args.steps} quarter-frame samples, OpenMP on {os.cpu_count()} threads; the "
                                   "reference's own CPU device is a software Vulkan renderer (unavailable on this "
                                   "box) and its Rust crate cannot be built here, so the oracle port stands in"},
        "e2e": {"value": round(v, 4), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_once() -> None:
    """One luma NLM launch of the workload (1920x1080, d=2, a=5, s=2): the small case the kernel
    profiles are captured on (three pushes fill the window once; ~60 MB on the device)."""
    import numpy as np
    import torch

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import synth

    clip = synth.make_clip(W, H, 3, depth=8, chroma="gray", sigma_luma=8.0, global_motion=4, sprites=3, seed=7)
    fmt = avd.SampleFormat.u8()
    t = avd.NlmTuning(search_radius=LUMA["a"], patch_radius=LUMA["s"], strength=LUMA["strength"])
    alg = avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=t, mode=avd.DenoisingMode.temporal(LUMA["d"])))
    eng = avd.build_engine(avd.EngineSpec.nlmeans(alg, None, avd.Geometry(W, H, avd.ChromaLayout.GRAY, fmt, fmt)))
    out = torch.zeros(plane_words(fmt, W, H), dtype=torch.int32, device="cuda")
    bufs = []
    for f in clip:
        flat = f[0].reshape(-1)
        b = torch.from_numpy(np.concatenate([flat, np.zeros((-flat.size) % 4, np.uint8)]).view(np.int32)).cuda()
        bufs.append(b)
        if eng.push([avd.DevicePlane.from_tensor(b, W, H)]):
            eng.emit_into([avd.DevicePlane.from_tensor(out, W, H)])
    torch.cuda.synchronize()
    eng.close()
    print("one luma NLM launch done")


def run_host(frames: int) -> None:
    """The host denoiser (wire bytes in, wire bytes out) against the same engine fed from HBM:
    1920x1080 4:2:0 u8, luma NLMeans d=2 a=5 s=2 strength 8, chroma passed through. Pushes
    `frames` frames with the push/recv pattern of the reference's host API and a flush, timed by the
    host clock from the first push to the last frame handed back; the resident run times the same
    pushes and emits with CUDA events. Prints one JSON line."""
    import numpy as np
    import torch

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import synth

    clip = synth.temporal_1080p_clip(frames=8, seed=11)
    fmt = avd.SampleFormat.u8()
    t = avd.NlmTuning(search_radius=LUMA["a"], patch_radius=LUMA["s"], strength=LUMA["strength"])
    alg = avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=t, mode=avd.DenoisingMode.temporal(LUMA["d"])))
    spec = avd.EngineSpec.nlmeans(alg, None, avd.Geometry(W, H, avd.ChromaLayout.YUV420, fmt, fmt))
    wire = [[np.ascontiguousarray(p).tobytes() for p in f] for f in clip]

    sinks = [bytearray(len(b)) for b in wire[0]]

    def host_pass(den, lockstep):
        """lockstep: `recv` (a fresh buffer set) after every push, the reference's doc example;
        pipelined: `recv_into` caller-owned buffers only when the queue is full, keeping
        MAX_PENDING frames in flight."""
        got = 0
        for k in range(frames):
            planes = wire[k % len(wire)]
            try:
                den.push(planes)
            except avd.QueueFull:
                got += den.recv() is not None if lockstep else den.recv_into(sinks)
                den.push(planes)
            if lockstep and den.recv() is not None:
                got += 1
        out = []
        den.flush(out.append)
        return got + len(out)

    host_times, host_split = {}, {}
    for lockstep in (False, True):
        den = avd.HostDenoiser(spec)
        host_pass(den, lockstep)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            n = host_pass(den, lockstep)
            ts.append(time.perf_counter() - t0)
            assert n == frames
        name = "lockstep" if lockstep else "pipelined"
        host_times[name] = ts
        tm = den.timing()
        per = 1e3 / max(1, tm.frames)
        host_split[name] = {"blocked_ms_per_frame": round(tm.blocked * per, 4),
                            "submit_ms_per_frame": round(tm.submit * per, 4),
                            "outside_calls_ms_per_frame": round((4 * sum(ts) / 3 * 1e3) / max(1, tm.frames)
                                                                - (tm.blocked + tm.submit) * per, 4)}
        den.close()

    dims = [spec.geometry.plane_dims(i) for i in range(3)]
    eng = avd.build_engine(spec)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    dev = [[torch.from_numpy(np.frombuffer(b + bytes((-len(b)) % 4), np.int32).copy()).cuda() for b in f]
           for f in wire]
    outb = [torch.zeros(plane_words(fmt, w, h), dtype=torch.int32, device="cuda") for (w, h) in dims]
    planes = [[avd.DevicePlane.from_tensor(b, w, h) for b, (w, h) in zip(f, dims)] for f in dev]
    out_planes = [avd.DevicePlane.from_tensor(b, w, h) for b, (w, h) in zip(outb, dims)]

    def device_pass():
        for k in range(frames):
            for _ in range(eng.push(planes[k % len(planes)])):
                eng.emit_into(out_planes)
        for _ in range(eng.finish()):
            eng.emit_into(out_planes)

    device_pass()
    torch.cuda.synchronize()
    dev_times = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        device_pass()
        e1.record(stream)
        torch.cuda.synchronize()
        dev_times.append(e0.elapsed_time(e1) / 1e3)
    eng.close()
    wire_bytes = sum(len(b) for b in wire[0])
    dev_fps = frames / statistics.median(dev_times)
    line = {"workload": "host denoiser: 1920x1080 4:2:0 u8, luma NLMeans d=2 a=5 s=2 strength 8, chroma passthrough",
            "frames": frames, "resident_frames_per_s": round(dev_fps, 2),
            "wire_bytes_per_frame_each_way": wire_bytes, "resident_ms": [round(x * 1e3, 2) for x in dev_times]}
    for name, ts in host_times.items():
        fps = frames / statistics.median(ts)
        line[name] = {"frames_per_s": round(fps, 2), "over_resident": round(fps / dev_fps, 4),
                      "ms": [round(x * 1e3, 2) for x in ts], **host_split[name]}
    print(json.dumps(line))


def run_prefilters(pushes: int) -> None:
    """The NLMeans prefilters on the headline luma pass: 1920x1080 u8 luma, d=2, a=5, s=2,
    strength 8, once with no prefilter, once with the bilateral reference ring (sigma_s 1.5, sigma_r
    0.05: a 7x7 kernel) and once with the spatial-NLM pilot (strength scale 0.4). Each push writes one
    ring slot (and its reference) and denoises one frame; prints the steady-state device time per
    frame of each (CUDA events around every push) as one JSON line."""
    import numpy as np
    import torch

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import synth

    clip = synth.temporal_1080p_clip(frames=8, seed=21)
    fmt = avd.SampleFormat.u8()
    stream = torch.cuda.current_stream()
    bufs = []
    for f in clip:
        flat = f[0].reshape(-1)
        bufs.append(torch.from_numpy(np.concatenate([flat, np.zeros((-flat.size) % 4, np.uint8)]).view(np.int32)).cuda())
    out = torch.zeros_like(bufs[0])
    res = {}
    for name, pf in (("none", avd.PrefilterMode.none()), ("bilateral:1.5,0.05", avd.PrefilterMode.bilateral(1.5, 0.05)),
                     ("nlm:0.4", avd.PrefilterMode.nlm_spatial(0.4))):
        t = avd.NlmTuning(search_radius=LUMA["a"], patch_radius=LUMA["s"], strength=LUMA["strength"])
        alg = avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(prefilter=pf, tuning=t,
                                                           mode=avd.DenoisingMode.temporal(LUMA["d"])))
        eng = avd.build_engine(avd.EngineSpec.nlmeans(alg, None, avd.Geometry(W, H, avd.ChromaLayout.GRAY, fmt, fmt)))
        eng.set_stream(stream.cuda_stream)
        times = []
        for i in range(pushes):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if eng.push([avd.DevicePlane.from_tensor(bufs[i % len(bufs)], W, H)]):
                eng.emit_into([avd.DevicePlane.from_tensor(out, W, H)])
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        eng.close()
        steady = times[2 * LUMA["d"] + 1:]
        res[name] = round(float(np.median(steady)), 4)
    print(json.dumps({"workload": "NLMeans 1920x1080 u8 luma d=2 a=5 s=2 strength 8, per prefilter",
                      "ms_per_frame": res,
                      "over_plain": {k: round(v / res["none"], 4) for k, v in res.items()}}))


def run_motion_compensated(pushes: int) -> None:
    """NLMeans with motion compensation on the headline luma pass: 1920x1080 u8 luma, d=2, a=5, s=2,
    strength 8, default motion search (blksize 16, overlap 8, radius 4, 2 levels, Direct at d=2 with
    the truemotion stage), plain, with escalation to 8, and NLMeans-HQ with a pinned sigma and
    temporal confidence.
    Prints the steady-state device time per frame of each as one JSON line."""
    import numpy as np
    import torch

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import synth

    clip = synth.temporal_1080p_clip(frames=8, seed=21)
    fmt = avd.SampleFormat.u8()
    stream = torch.cuda.current_stream()
    bufs = []
    for f in clip:
        flat = f[0].reshape(-1)
        bufs.append(torch.from_numpy(np.concatenate([flat, np.zeros((-flat.size) % 4, np.uint8)]).view(np.int32)).cuda())
    out = torch.zeros_like(bufs[0])
    t = avd.NlmTuning(search_radius=LUMA["a"], patch_radius=LUMA["s"], strength=LUMA["strength"])
    mode = avd.DenoisingMode.temporal(LUMA["d"])
    mc = avd.MotionCompensationMode(avd.MotionSearch())
    # The slow presets' search: failing blocks widen from radius 4 to 8 (motion/escalate.rs).
    mc_slow = avd.MotionCompensationMode(avd.MotionSearch(max_search_escalation=8))
    cases = {
        "plain": avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=t, mode=mode)),
        "motion compensated": avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(motion_compensation=mc, tuning=t,
                                                                           mode=mode)),
        "motion compensated, escalation to 8": avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(
            motion_compensation=mc_slow, tuning=t, mode=mode)),
        "HQ pinned sigma 8 codes, confidence, motion compensated": avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(
            nlm=avd.NlmeansOptions(motion_compensation=mc, tuning=avd.NlmTuning(search_radius=LUMA["a"],
                                                                               patch_radius=LUMA["s"]), mode=mode),
            hq=avd.HqParams(sigma_override=8.0 / 255.0))),
    }
    res = {}
    for name, alg in cases.items():
        eng = avd.build_engine(avd.EngineSpec.nlmeans(alg, None, avd.Geometry(W, H, avd.ChromaLayout.GRAY, fmt, fmt)))
        eng.set_stream(stream.cuda_stream)
        times = []
        for i in range(pushes):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if eng.push([avd.DevicePlane.from_tensor(bufs[i % len(bufs)], W, H)]):
                eng.emit_into([avd.DevicePlane.from_tensor(out, W, H)])
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        eng.close()
        res[name] = round(float(np.median(times[2 * LUMA["d"] + 1:])), 4)
    print(json.dumps({"workload": "NLMeans 1920x1080 u8 luma d=2 a=5 s=2 strength 8, motion compensation",
                      "ms_per_frame": res}))


def run_hq_auto(pushes: int, prefilter: str = "none") -> None:
    """NLMeans-HQ with the automatic noise estimate: 1920x1080 u8 luma, d=2, a=5, s=2, default HQ
    strength and temporal confidence, on the 1080p temporal clip. Each push reads one frame's noise
    in the look-ahead (Immerkaer, temporal records, reading) and, once the look-ahead and the ring
    are full, folds the window and denoises one frame. Prints the device time of every push (CUDA
    events) and the steady-state median as one JSON line."""
    import numpy as np
    import torch

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import synth

    clip = synth.temporal_1080p_clip(frames=8, seed=21)
    fmt = avd.SampleFormat.u8()
    t = avd.NlmTuning(search_radius=LUMA["a"], patch_radius=LUMA["s"])
    hq = avd.HqParams(sigma_override=None)
    alg = avd.NlmeansAlgorithm.hq_(avd.NlmeansHqOptions(
        nlm=avd.NlmeansOptions(prefilter=avd.parse_prefilter(prefilter), tuning=t,
                               mode=avd.DenoisingMode.temporal(LUMA["d"])), hq=hq))
    eng = avd.build_engine(avd.EngineSpec.nlmeans(alg, None, avd.Geometry(W, H, avd.ChromaLayout.GRAY, fmt, fmt)))
    stream = torch.cuda.current_stream()
    eng.set_stream(stream.cuda_stream)
    bufs = []
    for f in clip:
        flat = f[0].reshape(-1)
        bufs.append(torch.from_numpy(np.concatenate([flat, np.zeros((-flat.size) % 4, np.uint8)]).view(np.int32)).cuda())
    out = torch.zeros_like(bufs[0])
    times = []
    for i in range(pushes):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if eng.push([avd.DevicePlane.from_tensor(bufs[i % len(bufs)], W, H)]):
            eng.emit_into([avd.DevicePlane.from_tensor(out, W, H)])
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    eng.close()
    steady = times[8 + 2 * LUMA["d"] + 1:]
    ms = float(np.median(steady)) if steady else float("nan")
    print(json.dumps({"workload": "NLMeans-HQ automatic sigma, 1920x1080 u8 luma, d=2 a=5 s=2, temporal confidence",
                      "prefilter": prefilter,
                      "ms_per_frame": round(ms, 4), "frames_per_s": round(1000.0 / ms, 2),
                      "push_ms": [round(x, 3) for x in times]}))


def run_nl4d(pushes: int, size: str) -> None:
    """The NL4D engine on one plane of synthetic content with a pinned sigma and Direct motion:
    1920x1080 u8 or 3840x2160 10-bit luma, d=2, spatial radius 9, defaults otherwise. Prints the
    device time of every push (CUDA events on the engine's stream) and the steady-state median as
    one JSON line. The first 2d+1 pushes fill the ring (the last of them runs d+1 passes)."""
    import numpy as np
    import torch

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import synth

    w, h, depth = (1920, 1080, 8) if size == "1080" else (3840, 2160, 10)
    d = 2
    fmt = avd.SampleFormat.u8() if depth == 8 else avd.SampleFormat.u16(depth)
    o = avd.Nl4dOptions(sigma=10.0 / 255, temporal_radius=d, spatial_radius=9,
                        motion=avd.MotionSearch(estimation=avd.MotionEstimation.DIRECT))
    eng = avd.build_engine(avd.EngineSpec.nl4d(o, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt)))
    stream = torch.cuda.current_stream()
    eng.set_stream(stream.cuda_stream)
    clip = synth.make_clip(w, h, 4, depth=depth, chroma="gray", sigma_luma=10.0, global_motion=2, sprites=3,
                           sprite_size=200, seed=1)
    dt = np.uint8 if depth == 8 else np.uint16
    bufs = []
    for f in clip:
        flat = f[0].reshape(-1).astype(dt)
        spw = 4 if depth == 8 else 2
        bufs.append(torch.from_numpy(np.concatenate([flat, np.zeros((-flat.size) % spw, dt)]).view(np.int32)).cuda())
    out = torch.zeros_like(bufs[0])
    times = []
    for i in range(pushes):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ready = eng.push([avd.DevicePlane.from_tensor(bufs[i % 4], w, h)])
        for _ in range(ready):
            eng.emit_into([avd.DevicePlane.from_tensor(out, w, h)])
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    eng.close()
    steady = times[2 * d + 1:]
    ms = float(np.median(steady)) if steady else float("nan")
    print(json.dumps({"workload": f"NL4D {w}x{h} luma u{depth} d=2 spatial_radius 9 pinned sigma, Direct motion",
                      "ms_per_frame": round(ms, 4), "frames_per_s": round(1000.0 / ms, 2) if steady else None,
                      "push_ms": [round(t, 3) for t in times]}))


def run_nl4d_4k(pushes: int, auto: bool = False, wiener: bool = False) -> None:
    """NL4D on the 4K workload: 3840x2160 4:2:0 10-bit, 7-frame window (d=3, Auto estimation resolves
    to Chained), spatial radius 16, hard threshold 2.7 (lambda_ht 2.7, scale 1, pooled threshold and
    noise map off), motion at its defaults. Synthetic frames: the gratings/rectangles/texture base in
    10-bit codes, 12 sprites at integer velocities up to 8 px/frame, Gaussian noise of 20 codes plus
    signal-dependent variance 0.02 * value. Eight generated frames are cycled.

    Default: luma and chroma in one engine with sigma pinned at 20 codes. With `auto`, both plane
    groups take their sigma from the automatic noise estimate (motion-compensated look-ahead) with the
    luma noise map and the colour grain gains on, the reference's defaults. With `wiener`, every pass
    adds the empirical Wiener stage after the threshold. Prints the device time of every push and the
    steady-state median as one JSON line."""
    import numpy as np
    import torch

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import synth

    w, h, depth, d = 3840, 2160, 10, 3
    fmt = avd.SampleFormat.u16(depth)
    sigma = 20.0 / 1023.0

    def options(sig):
        return avd.Nl4dOptions(sigma=sig, temporal_radius=d, spatial_radius=16, lambda_ht=2.7, lambda_ht_scale=1.0,
                               pooled_threshold=False, noise_map=sig is None, wiener=wiener)

    geo = avd.Geometry(w, h, avd.ChromaLayout.YUV420, fmt, fmt)
    o = options(None if auto else sigma)
    engines = [avd.build_engine(avd.EngineSpec.nl4d(o, o, geo))]
    stream = torch.cuda.current_stream()
    for eng in engines:
        eng.set_stream(stream.cuda_stream)
    clip = synth.make_clip(w, h, 8, depth=depth, chroma="420", sigma_luma=20.0 / 4.0, sigma_chroma=20.0 / 4.0,
                           sprites=12, sprite_speed=8, signal_dependent=0.02, seed=2000)
    dims = [geo.plane_dims(i) for i in range(3)]
    bufs = []
    for f in clip:
        planes = []
        for p, (pw, ph) in zip(f, dims):
            flat = p.reshape(-1).astype(np.uint16)
            planes.append(torch.from_numpy(np.concatenate([flat, np.zeros(flat.size % 2, np.uint16)]).view(np.int32)).cuda())
        bufs.append(planes)
    outs = [torch.zeros_like(b) for b in bufs[0]]

    def dp(ts):
        return [avd.DevicePlane.from_tensor(t, pw, ph) for t, (pw, ph) in zip(ts, dims)]

    times = []
    for i in range(pushes):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for eng in engines:
            ready = eng.push(dp(bufs[i % len(bufs)]))
            for _ in range(ready):
                eng.emit_into(dp(outs))
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    for eng in engines:
        eng.close()
    warm = 2 * d + 1 + (8 if auto else 0)
    steady = times[warm:]
    ms = float(np.median(steady))
    what = ("sigma from the automatic noise estimate on both plane groups, noise map and colour gains on" if auto
            else "sigma pinned at 20 codes") + (", Wiener stage" if wiener else "")
    print(json.dumps({"workload": "NL4D 3840x2160 4:2:0 10-bit luma+chroma, d=3 (Chained), spatial_radius 16, "
                                  "lambda_ht 2.7, plain threshold, " + what,
                      "ms_per_frame": round(ms, 3), "frames_per_s": round(1000.0 / ms, 2),
                      "push_ms": [round(t, 2) for t in times]}))


def run_adjoint(reps: int) -> None:
    """The NLMeans adjoint (`avd_nlm_backward`) against its forward on the same window: 1920x1080
    luma, d=2, a=5, s=2, strength 8, fast variant. The forward is the engine's push (ingest + the
    windowed NLM launch) in steady state; both are timed with CUDA events on one stream. Prints one
    JSON line with both times and their ratio."""
    import ctypes as C

    import numpy as np
    import torch

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import _abi, synth

    lib = _abi.load()
    w, h, d, a, s, strength = W, H, 2, 5, 2, 8.0
    fmt = avd.SampleFormat.u8()
    clip = synth.make_clip(w, h, 2 * d + 1, depth=8, chroma="gray", sigma_luma=8.0, global_motion=4, sprites=3,
                           seed=7)
    t = avd.NlmTuning(search_radius=a, patch_radius=s, strength=strength)
    alg = avd.NlmeansAlgorithm.fast(avd.NlmeansOptions(tuning=t, mode=avd.DenoisingMode.temporal(d)))
    eng = avd.build_engine(avd.EngineSpec.nlmeans(alg, None, avd.Geometry(w, h, avd.ChromaLayout.GRAY, fmt, fmt)))
    stream = torch.cuda.current_stream()
    eng.set_stream(stream.cuda_stream)
    bufs = []
    for f in clip:
        flat = f[0].reshape(-1)
        bufs.append(torch.from_numpy(np.concatenate([flat, np.zeros((-flat.size) % 4, np.uint8)]).view(np.int32)).cuda())
    out = torch.zeros_like(bufs[0])

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def push(i):
        if eng.push([avd.DevicePlane.from_tensor(bufs[i % len(bufs)], w, h)]):
            eng.emit_into([avd.DevicePlane.from_tensor(out, w, h)])

    for i in range(3):
        push(i)
    fwd = [timed(lambda i=i: push(i)) for i in range(3, 3 + reps)]
    eng.close()
    window = torch.from_numpy(np.stack([f[0].astype(np.float32) / 255.0 for f in clip]).reshape(-1)).cuda()
    g = torch.randn(w * h, device="cuda")
    gw = torch.empty_like(window)
    gs = torch.zeros(1, device="cuda")
    scratch = torch.empty(lib.avd_nlm_backward_scratch_bytes(w, h) // 4, device="cuda")
    p = _abi.AvdNlmBackward()
    p.window, p.grad_out, p.grad_window, p.grad_strength = window.data_ptr(), g.data_ptr(), gw.data_ptr(), gs.data_ptr()
    p.scratch = scratch.data_ptr()
    p.width, p.height, p.channels, p.temporal_radius, p.search_radius, p.patch_radius = w, h, 1, d, a, s
    p.strength, p.self_weight, p.pair_offset, p.spatial_offset = strength, 1.0, 0.0, 0.0

    def backward():
        st = lib.avd_nlm_backward(C.byref(p), C.c_void_p(stream.cuda_stream))
        if st != 0:
            raise RuntimeError(lib.avd_last_error().decode())

    backward()
    bwd = [timed(backward) for _ in range(reps)]
    f_ms, b_ms = float(np.median(fwd)), float(np.median(bwd))
    print(json.dumps({"workload": "NLMeans adjoint, 1920x1080 luma f32 window, d=2 a=5 s=2 strength 8",
                      "forward_ms": round(f_ms, 4), "backward_ms": round(b_ms, 4),
                      "backward_over_forward": round(b_ms / f_ms, 3)}))
    run_nl4d_adjoint(reps)


def run_nl4d_adjoint(reps: int) -> None:
    """The NL4D collab pass (`avd_collab_pass`: group search and filter) against its adjoint
    (`avd_collab_adjoint`) on one 1920x1080 luma window of 5 frames (temporal radius 2, spatial
    radius 9, refine 2, plain threshold 2.7 sigma, zero motion at full confidence), with and without
    the Wiener stage. CUDA events on one stream; the accumulators are cleared outside the timed
    region. One JSON line per setting."""
    import ctypes as C

    import numpy as np
    import torch

    import av_denoise_b200_loader

    av_denoise_b200_loader.load()
    from av_denoise_b200 import _abi, synth
    from av_denoise_b200.autograd import Nl4dPassConfig, _Nl4dState

    lib = _abi.load()
    w, h, d = W, H, 2
    clip = synth.make_clip(w, h, 2 * d + 1, depth=8, chroma="gray", sigma_luma=10.0, global_motion=0, sprites=3,
                           seed=9)
    window = torch.from_numpy(np.stack([f[0].astype(np.float32) / 255.0 for f in clip])[..., None].copy()).cuda()
    sigma = torch.tensor([10.0 / 255.0], device="cuda")
    stream = torch.cuda.current_stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    for wiener in (False, True):
        cfg = Nl4dPassConfig(radius=d, spatial_radius=9, refine=2, lambda_ht=2.7, wiener=wiener)
        st = _Nl4dState(window, sigma, cfg)
        grad_accum = torch.randn(st.accum.numel(), device="cuda")
        grad_wsum = torch.randn(st.wsum.numel(), device="cuda")
        grad_window = torch.zeros_like(window)
        grad_refs = torch.empty(st.refs, device="cuda")
        adj = _abi.AvdCollabAdjoint(grad_accum.data_ptr(), grad_wsum.data_ptr(), grad_window.data_ptr(),
                                    grad_refs.data_ptr())

        def backward():
            code = lib.avd_collab_adjoint(C.byref(st.p), C.byref(adj), C.c_void_p(stream.cuda_stream))
            if code != 0:
                raise RuntimeError(lib.avd_last_error().decode())

        fwd, bwd = [], []
        for i in range(reps + 2):
            st.accum.zero_()
            st.wsum.zero_()
            f = timed(st.run)
            grad_window.zero_()
            b = timed(backward)
            if i >= 2:
                fwd.append(f)
                bwd.append(b)
        f_ms, b_ms = float(np.median(fwd)), float(np.median(bwd))
        print(json.dumps({"workload": "NL4D collab pass adjoint, 1920x1080 luma window of 5 frames, spatial radius 9, "
                                      "refine 2, threshold 2.7" + (", Wiener stage" if wiener else ""),
                          "forward_ms": round(f_ms, 4), "backward_ms": round(b_ms, 4),
                          "backward_over_forward": round(b_ms / f_ms, 3)}))


def run_batch(reps: int) -> None:
    """The batched NLMeans launch against the plain per-frame loop on a mix of 24 clips: resolution
    from {640x360, 1280x720, 1920x1080, 2560x1440, 3840x2160}, depth from {8, 10, 12}, 4-17 frames,
    temporal radius 1-8, a=4, s=2, NLMeans-HQ with each clip's sigma pinned (U(4, 24) in 8-bit
    units: strength = hq_default_strength(luma, d) * sigma and the flat noise offset). Frames are
    synthetic (six gratings, a pan, Gaussian noise, quantised to the clip's depth) generated on the
    device; every frame of every clip is one job. Both arms are timed with CUDA events."""
    import ctypes as C

    import numpy as np
    import torch

    import av_denoise_b200_loader

    avd = av_denoise_b200_loader.load()
    from av_denoise_b200 import _abi

    lib = _abi.load()
    rng = np.random.default_rng(3000)
    a, s = 4, 2
    sizes = [(640, 360), (1280, 720), (1920, 1080), (2560, 1440), (3840, 2160)]
    jobs, keep, singles, pixels = [], [], [], 0
    ingest_items, ingest_pairs = [], []  # the clips' frames as words of their own depth, and where they land
    for i in range(24):
        w, h = sizes[int(rng.integers(0, 5))]
        depth = int(rng.choice([8, 10, 12]))
        n = int(rng.integers(4, 18))
        d = int(rng.integers(1, 9))
        sigma = float(rng.uniform(4.0, 24.0)) / 255.0
        y, x = torch.meshgrid(torch.arange(h, device="cuda", dtype=torch.float32),
                              torch.arange(w, device="cuda", dtype=torch.float32), indexing="ij")
        base = torch.zeros(h, w, device="cuda")
        for _ in range(6):
            f, th = float(rng.uniform(0.01, 0.3)), float(rng.uniform(0, np.pi))
            base += float(rng.uniform(5, 30)) / 255.0 * torch.sin(2 * np.pi * f * (x * np.cos(th) + y * np.sin(th)))
        base = (base + 0.5).clamp(16 / 255, 235 / 255)
        levels = float(2 ** depth - 1)
        gen = torch.Generator(device="cuda").manual_seed(1000 * 3 + i)
        frames = torch.stack([torch.roll(base, shifts=(int(rng.integers(-4, 5)) * t,), dims=(1,)) +
                              sigma * torch.randn(h, w, generator=gen, device="cuda") for t in range(n)])
        codes = (frames.clamp(0, 1) * levels).round()
        frames = codes / levels
        keep.append(frames)
        words = codes.to(torch.uint8 if depth == 8 else torch.int16).contiguous().view(torch.int32)
        landed = torch.empty_like(frames)
        keep += [words, landed]
        per_frame_words = words.numel() // n
        for t in range(n):
            ingest_items.append(_abi.AvdBatchIngest(words.data_ptr() + 4 * t * per_frame_words, 0,
                                                    landed.data_ptr() + 4 * t * h * w, w, h, 1, depth))
        # the engine's ingest divides (correctly rounded); torch's division by a Python scalar
        # multiplies by its reciprocal, so the check divides by a tensor of the same shape
        ingest_pairs.append((codes / torch.full_like(codes, levels), landed))
        strength = float(avd.hq_default_strength(1, d)) * sigma * 255.0
        offset = float(np.float32(2.0 * 3.0) * np.float32(sigma) ** 2 * np.float32((2 * s + 1) ** 2))
        for c in range(n):
            out = torch.empty(h * w, device="cuda")
            keep.append(out)
            jobs.append(_abi.AvdBatchJob(frames.data_ptr(), out.data_ptr(), n, c, d, w, h, strength, offset, offset))
            singles.append((frames, c, d, strength, offset, out, w, h))
            pixels += w * h
    arr = (_abi.AvdBatchJob * len(jobs))(*jobs)
    scratch = torch.empty(lib.avd_batch_scratch_bytes(len(jobs), a) // 4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    win_scratch = torch.empty(lib.avd_nlm_window_scratch_bytes(a) // 4 + 1, device="cuda")
    max_window = max(fr.shape[1] * fr.shape[2] * (2 * d + 1) for fr, _, d, *_ in singles)
    win_buf = torch.empty(max_window, device="cuda")

    def batched():
        if lib.avd_batch_submit(arr, len(jobs), 1, a, s, 1.0, scratch.data_ptr(), C.c_void_p(stream.cuda_stream)):
            raise RuntimeError(lib.avd_last_error().decode())

    params = []
    for frames, c, d, strength, offset, out, w, h in singles:
        n = frames.shape[0]
        idx = torch.tensor([min(max(c - d + k, 0), n - 1) for k in range(2 * d + 1)], device="cuda")
        p = _abi.AvdNlmBackward()
        p.window, p.grad_out, p.scratch = win_buf.data_ptr(), out.data_ptr(), win_scratch.data_ptr()
        p.width, p.height, p.channels, p.temporal_radius, p.search_radius, p.patch_radius = w, h, 1, d, a, s
        p.strength, p.self_weight, p.pair_offset, p.spatial_offset = strength, 1.0, offset, offset
        params.append((frames, idx, p, (2 * d + 1) * w * h))

    def per_frame():
        # The plain loop: one windowed launch per frame (the window gathered into one buffer, as a
        # per-clip ring holds it).
        for frames, idx, p, count in params:
            torch.index_select(frames, 0, idx, out=win_buf[:count].view(idx.numel(), *frames.shape[1:]))
            if lib.avd_nlm_window(C.byref(p), C.c_void_p(stream.cuda_stream)):
                raise RuntimeError(lib.avd_last_error().decode())

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    batched()
    per_frame()
    b_ms = float(np.median([timed(batched) for _ in range(reps)]))
    l_ms = float(np.median([timed(per_frame) for _ in range(reps)]))
    # The clips' 8-, 10- and 12-bit words normalised in one launch (`avd_batch_ingest`).
    iarr = (_abi.AvdBatchIngest * len(ingest_items))(*ingest_items)
    iscratch = torch.empty(lib.avd_batch_ingest_scratch_bytes(len(ingest_items)) // 4 + 1, dtype=torch.int32,
                           device="cuda")

    def ingest():
        if lib.avd_batch_ingest(iarr, len(ingest_items), iscratch.data_ptr(), C.c_void_p(stream.cuda_stream)):
            raise RuntimeError(lib.avd_last_error().decode())

    ingest()
    torch.cuda.synchronize()
    ingest_same = all(torch.equal(f, g) for f, g in ingest_pairs)
    i_ms = float(np.median([timed(ingest) for _ in range(reps)]))
    print(json.dumps({"workload": f"NLMeans-HQ pinned sigma, 24 mixed clips, {len(jobs)} frames, "
                                  f"{pixels / 1e6:.1f} Mpixel, a=4 s=2, d 1-8",
                      "batched_ms": round(b_ms, 3), "per_frame_loop_ms": round(l_ms, 3),
                      "speedup": round(l_ms / b_ms, 3),
                      "batched_frames_per_s": round(len(jobs) / b_ms * 1000.0, 2),
                      "batched_ingest_ms": round(i_ms, 3), "batched_ingest_frames": len(ingest_items),
                      "batched_ingest_matches_normalised_frames": bool(ingest_same)}))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--once", action="store_true", help="run one luma NLM launch (profiling case) and exit")
    ap.add_argument("--nl4d", type=int, default=0, metavar="PUSHES",
                    help="time PUSHES pushes of the NL4D engine (secondary workload) and exit")
    ap.add_argument("--nl4d-size", default="1080", choices=["1080", "2160"])
    ap.add_argument("--nl4d-4k", type=int, default=0, metavar="PUSHES",
                    help="time PUSHES pushes of the 4K 4:2:0 10-bit NL4D workload (d=3) and exit")
    ap.add_argument("--wiener", action="store_true", help="with --nl4d-4k: the Wiener stage after the threshold")
    ap.add_argument("--auto-sigma", action="store_true",
                    help="with --nl4d-4k: sigma from the automatic noise estimate on both plane groups")
    ap.add_argument("--adjoint", type=int, default=0, metavar="REPS",
                    help="time the NLMeans adjoint against its forward REPS times and exit")
    ap.add_argument("--batch", type=int, default=0, metavar="REPS",
                    help="time the batched launch against the per-frame loop REPS times and exit")
    ap.add_argument("--host", type=int, default=0, metavar="FRAMES",
                    help="time FRAMES frames through the host denoiser against the resident engine and exit")
    ap.add_argument("--hq-auto", type=int, default=0, metavar="PUSHES",
                    help="time PUSHES pushes of NLMeans-HQ with the automatic noise estimate and exit")
    ap.add_argument("--prefilters", type=int, default=0, metavar="PUSHES",
                    help="time the headline luma pass with no prefilter, the bilateral and the NLM pilot")
    ap.add_argument("--mc", type=int, default=0, metavar="PUSHES",
                    help="time the headline luma pass with motion compensation (plain and HQ)")
    ap.add_argument("--prefilter", default="none", help="prefilter of --hq-auto (none, nlm[:scale], bilateral:ss,sr)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the parity frame and the CPU baseline")
    ap.add_argument("--no-nl4d", action="store_true", help="skip the NL4D 4K fields of the default line")
    ap.add_argument("--nl4d-pushes", type=int, default=30)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    args = ap.parse_args()
    if args.once:
        run_once()
    elif args.nl4d:
        run_nl4d(args.nl4d, args.nl4d_size)
    elif args.nl4d_4k:
        run_nl4d_4k(args.nl4d_4k, auto=args.auto_sigma, wiener=args.wiener)
    elif args.adjoint:
        run_adjoint(args.adjoint)
    elif args.batch:
        run_batch(args.batch)
    elif args.host:
        run_host(args.host)
    elif args.hq_auto:
        run_hq_auto(args.hq_auto, args.prefilter)
    elif args.prefilters:
        run_prefilters(args.prefilters)
    elif args.mc:
        run_motion_compensated(args.mc)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
