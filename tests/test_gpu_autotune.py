"""Autotuner on the GPU: tuning times the candidates, caches the winner per
(device, build, shape, table mode, segment length, bits per weight, batch) in the
JSON file, reuses it without timing, and the tuned launch is bit-exact."""
import numpy as np
import pytest

from conftest import cuda_ok
import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ok(), reason="needs a CUDA device")]

if cuda_ok():
    import torch
    from matvans_b200 import autotune, ops


def test_tune_caches_and_reuses(tmp_path, monkeypatch):
    monkeypatch.setenv("MATVANS_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(12)
    W = np.clip(np.round(rng.normal(0, 4, size=(512, 1024))), -127, 127).astype(np.int8)
    M = ops.Q8Matrix.encode(W, local=True)
    cands = [(4, 1, 1, 0, 0, 0), (8, 2, 1, 0, 0, 0), (8, 1, 1, 0, 2, 0)]
    t1, e1 = autotune.tune(M, batch=1, candidates=cands, reps=2)
    assert sorted(e1["all"]) == sorted(",".join(map(str, c)) for c in cands)
    assert tuple(e1["tuning"]) in cands and e1["us"] == min(e1["all"].values())

    calls = []
    real = autotune.time_launches
    monkeypatch.setattr(autotune, "time_launches", lambda *a, **k: calls.append(1) or real(*a, **k))
    t2, e2 = autotune.tune(M, batch=1, candidates=cands, reps=2)
    assert not calls and e2 == e1                     # served from the cache
    t16, e16 = autotune.tune(M, batch=16, reps=2)     # another key: timed, both engines
    assert calls and any(k.endswith(",1") for k in e16["all"]) and any(k.endswith(",0") for k in e16["all"])
    calls.clear()
    autotune.tune(M, batch=1, candidates=cands, reps=2, force=True)
    assert calls

    for t, B in ((t1, 1), (t16, 16)):
        x = rng.integers(-127, 128, size=(B, 1024)).astype(np.int8)
        assert np.array_equal(M.matvec(torch.from_numpy(x), tuning=t).cpu().numpy(), oracle.matvec_i8(W, x))
    assert ops.device_status() == 0


def test_tune_stack_picks_a_launchable_candidate():
    rng = np.random.default_rng(13)
    Ms = [ops.Q8Matrix.encode(np.clip(np.round(rng.normal(0, 3, size=sh)), -127, 127).astype(np.int8))
          for sh in ((256, 512), (512, 256))]
    best, res = autotune.tune_stack(lambda t: ops.Q8Stack(Ms, batch=8, tuning=t),
                                    candidates=autotune.candidates_for(8, autotune.CANDIDATES), reps=2)
    assert ",".join(map(str, best)) in res and len(res) >= 8
    assert ops.device_status() == 0


def test_tune_stack_caches_by_stack_key(tmp_path, monkeypatch):
    monkeypatch.setenv("MATVANS_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(14)
    Ws = [np.clip(np.round(rng.normal(0, 3, size=sh)), -127, 127).astype(np.int8) for sh in ((256, 512), (96, 1024))]
    Ms = [ops.Q8Matrix.encode(W) for W in Ws]
    key = autotune.stack_key(Ms, 1)
    assert key != autotune.stack_key(Ms, 4) and key != autotune.stack_key(Ms[::-1], 1)
    built = []
    make = lambda t: built.append(t) or ops.Q8Stack(Ms, batch=1, tuning=t)  # noqa: E731
    cands = [(4, 1, 1, 0, 0, 0), (8, 2, 1, 0, 0, 0), (16, 1, 1, 0, 0, 0)]
    best, res = autotune.tune_stack(make, candidates=cands, reps=2, key=key)
    assert len(built) == 3 and best in cands
    built.clear()
    best2, res2 = autotune.tune_stack(make, candidates=cands, reps=2, key=key)
    assert not built and best2 == best and res2 == res  # served from the cache
    xs = [torch.from_numpy(rng.integers(-127, 128, size=(1, W.shape[1])).astype(np.int8)).cuda() for W in Ws]
    S = ops.Q8Stack(Ms, batch=1, tuning=best2, xs=xs)
    S.run()
    for W, x, y in zip(Ws, xs, S.ys):
        assert np.array_equal(y.cpu().numpy(), oracle.matvec_i8(W, x.cpu().numpy()))
    assert ops.device_status() == 0
