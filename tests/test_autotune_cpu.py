"""Autotuner host logic (no GPU): the candidate sets per batch and the JSON
cache (keys kept across processes that write at the same time, damaged files
read as empty)."""
import json
import multiprocessing as mp
import os

from matvans_b200 import autotune


def test_candidates_per_batch():
    base = autotune.SINGLE_CANDIDATES
    assert autotune.candidates_for(1, base) == list(base)
    assert autotune.candidates_for(2, base) == list(base)   # one or two vectors: the CUDA cores only
    for B in (3, 4, 8, 16):                                  # from 3 vectors on: both engines
        cb = autotune.candidates_for(B, base)
        mma = [c for c in cb if c[5] == 0]
        dp4a = [c for c in cb if c[5] == 1]
        assert mma and dp4a
        assert all(c[1] == 1 for c in mma)                   # the tensor-core engine decodes with ilp 1
        assert {c[0] for c in mma} == {4, 6, 8}              # up to 8 warps per CTA there
        assert sorted(c[:5] for c in dp4a) == sorted(c[:5] for c in base)  # every base candidate on CUDA cores
        assert len(set(cb)) == len(cb)


def test_cache_round_trip_and_damaged_file(tmp_path, monkeypatch):
    p = tmp_path / "sub" / "cache.json"
    monkeypatch.setenv("MATVANS_AUTOTUNE_CACHE", str(p))
    assert autotune._load() == {}
    autotune._update("k1", {"tuning": [8, 1, 1, 0, 0, 0], "us": 1.5})
    autotune._update("k2", {"tuning": [4, 2, 1, 0, 2, 0], "us": 2.5})
    db = json.loads(p.read_text())
    assert db["k1"]["us"] == 1.5 and db["k2"]["tuning"] == [4, 2, 1, 0, 2, 0]
    p.write_text("{ not json")
    assert autotune._load() == {}


def _writer(path, tag, n):
    os.environ["MATVANS_AUTOTUNE_CACHE"] = path
    from matvans_b200 import autotune as at
    for i in range(n):
        at._update(f"{tag}-{i}", {"tuning": [8, 1, 1, 0, 0, 0], "us": float(i)})


def test_concurrent_writers_keep_every_entry(tmp_path):
    path = str(tmp_path / "cache.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_writer, args=(path, t, 25)) for t in ("a", "b", "c")]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    db = json.load(open(path))
    assert sorted(db) == sorted(f"{t}-{i}" for t in "abc" for i in range(25))
