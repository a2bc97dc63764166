"""The launch tuner's choice and store on the CPU (tune/store.rs, driver/mod.rs, config.rs:8-75),
through `avd_tune_variant_for_test`, which times variant v as the given milliseconds instead of a
launch: Auto keeps the fastest (the baseline keeps ties) and writes one JSON line per key, Cached
reads the store and otherwise answers the baseline, Off always answers the baseline, and a later
process (the remembered results dropped) reads the stored choice without timing again."""

import ctypes as C
import json

import pytest

AUTO, CACHED, OFF = 0, 1, 2


def pick(lib, mode, store, key, times):
    arr = (C.c_float * len(times))(*times)
    return lib.avd_tune_variant_for_test(mode, store.encode() if store else None, key.encode(), len(times), arr)


@pytest.fixture
def store(tmp_path, lib):
    lib.avd_tune_forget()
    yield str(tmp_path)
    lib.avd_tune_forget()


def lines(path):
    with open(path + "/av-denoise-b200-tune.jsonl") as f:
        return [json.loads(line) for line in f if line.strip()]


def test_auto_keeps_the_fastest_and_stores_it(lib, store):
    assert pick(lib, AUTO, store, "site a", [1.0, 0.7, 0.9]) == 1
    rows = lines(store)
    assert len(rows) == 1 and rows[0]["format"] == 1 and rows[0]["variant"] == 1
    assert rows[0]["key"].endswith("site a") and rows[0]["ms"] == pytest.approx([1.0, 0.7, 0.9])
    # Remembered: asked again with other timings, the first answer stands and nothing is appended.
    assert pick(lib, AUTO, store, "site a", [0.1, 5.0, 5.0]) == 1
    assert len(lines(store)) == 1


def test_the_baseline_keeps_ties_and_failed_variants_are_skipped(lib, store):
    assert pick(lib, AUTO, store, "tie", [0.5, 0.5, 0.6]) == 0
    assert pick(lib, AUTO, store, "failed", [-1.0, 0.8, 0.4]) == 2
    assert pick(lib, AUTO, store, "all failed", [-1.0, -1.0]) == 0


def test_cached_reads_the_store_of_an_earlier_process(lib, store):
    assert pick(lib, AUTO, store, "shape", [2.0, 1.0, 3.0]) == 1
    lib.avd_tune_forget()  # a new process: only the file remains
    assert pick(lib, CACHED, store, "shape", [0.1, 9.0, 9.0]) == 1
    assert pick(lib, CACHED, store, "unknown shape", [9.0, 0.1]) == 0
    assert len(lines(store)) == 1


def test_off_and_single_variant_sites_answer_the_baseline(lib, store):
    assert pick(lib, OFF, store, "off", [9.0, 0.1]) == 0
    assert pick(lib, AUTO, store, "one", [9.0]) == 0
    import os

    assert not os.path.exists(store + "/av-denoise-b200-tune.jsonl")


def test_without_a_store_results_last_for_the_process(lib, store):
    assert pick(lib, AUTO, None, "memory", [3.0, 1.0]) == 1
    assert pick(lib, CACHED, None, "memory", [0.1, 9.0]) == 1
    lib.avd_tune_forget()
    assert pick(lib, CACHED, None, "memory", [0.1, 9.0]) == 0


def test_tuning_config_maps_onto_the_abi():
    from conftest import avd

    t = avd.TuningConfig(mode="cached", store="/tmp/x")._c()
    assert t.mode == CACHED and t.store == b"/tmp/x" and t.deterministic == 0
    with pytest.raises(avd.InvalidOptions):
        avd.TuningConfig(mode="sometimes")._c()
