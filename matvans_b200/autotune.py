"""Per-shape launch-parameter autotuner for the persistent Q8 kernel, with a JSON cache.

The tunables are the ones the kernel exposes through mv_q8_tuning: warps per
CTA, independent streams decoded per warp (ilp) and shared-memory stream buffer
depth (depth).  Stream interleave inside a row (segment length) is fixed when a
matrix is encoded (q8_encode's seg_quads), so it is part of the cache key.

Each candidate is timed as a CUDA graph of R launches over R copies of the
matrix, enough copies that their compressed bytes exceed twice the L2, so every
launch reads HBM as in real use.  The best candidate is cached under a key of
GPU name, driver, library build, shape, table mode, segment length, bits per
weight and batch, in $MATVANS_AUTOTUNE_CACHE (default
~/.cache/matvans_b200/autotune.json).
"""
import fcntl
import json
import os
import threading

import numpy as np
import torch

from . import _lib
from ._lib import Q8Tuning

# (warps, ilp, depth, ctas_per_sm, parts, engine)
CANDIDATES = [(w, ilp, d, 0, 0, 0) for w in (4, 8, 16) for ilp in (1, 2) for d in (1, 2)]
# single matrices additionally try splitting each stripe into more work items
SINGLE_CANDIDATES = CANDIDATES + [(w, ilp, d, 0, p, 0) for w in (4, 8) for ilp in (1, 2) for d in (1, 2)
                                  for p in (2, 4)]


def candidates_for(batch, base):
    """Candidates at `batch` vectors: from MMA_MIN_BATCH (3) vectors on they run
    on the tensor cores (engine 0, where ilp is fixed at 1) or on the CUDA cores
    (engine 1); fewer vectors always use the CUDA cores."""
    if batch < _lib.MMA_MIN_BATCH:
        return list(base)
    mma = sorted({(w, 1, c[2], c[3], c[4], 0) for c in base for w in (4, 6, 8)})  # at most 8 warps
    return mma + [c[:5] + (1,) for c in base]
L2_BYTES = 126 * 2 ** 20
_lock = threading.Lock()


def cache_path():
    return os.environ.get("MATVANS_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "matvans_b200", "autotune.json"))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(db):
    p = cache_path()
    os.makedirs(os.path.dirname(p) or ".", exist_ok=True)
    tmp = p + f".tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def _update(k, entry):
    """Adds one entry under an exclusive lock on <cache>.lock, so that processes tuning at the same time
    (one per GPU) keep each other's entries; the file itself is replaced atomically."""
    p = cache_path()
    os.makedirs(os.path.dirname(p) or ".", exist_ok=True)
    with _lock, open(p + ".lock", "a+") as lf:
        fcntl.flock(lf, fcntl.LOCK_EX)
        try:
            db = _load()
            db[k] = entry
            _store(db)
        finally:
            fcntl.flock(lf, fcntl.LOCK_UN)


def _build_id():
    st = os.stat(_lib.LIB_PATH)
    return f"{st.st_size}-{int(st.st_mtime)}"


def key(M, batch):
    props = torch.cuda.get_device_properties(M.device)
    drv = torch.cuda.get_device_capability(M.device)
    return (f"{props.name}|sm{drv[0]}{drv[1]}|{_build_id()}|{M.rows}x{M.cols}|local{M.local}|seg{M.seg_quads}"
            f"|bpw{M.bits_per_weight:.1f}|B{batch}")


def copies(M, n):
    """M and n - 1 device copies of its encoding (cold-L2 timing)."""
    from .ops import Q8Matrix
    enc = {"rows": M.rows, "cols": M.cols, "blocks": M.blocks.cpu().numpy(), "blk_off": M.blk_off.cpu().numpy(),
           "tbl": M.tbl.cpu().numpy().view(np.uint16), "tbl_off": M.tbl_off.cpu().numpy(),
           "seg_quads": M.seg_quads, "nseg": M.nseg, "local": M.local, "max_blk_rows": M.max_blk_rows,
           "tbl_stripe_max": M.tbl_stripe_max, "payload_bytes": M.payload_bytes,
           "bits_per_weight": M.bits_per_weight}
    return [M] + [Q8Matrix(enc, device=M.device) for _ in range(n - 1)]


def time_launches(fns, reps=10):
    """ms per call of each fn in `fns`, replayed as one CUDA graph."""
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for f in fns:
            f()
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for f in fns:
            f()
    g.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps / len(fns)


def tune(M, batch=1, candidates=None, reps=10, force=False):
    """Best Q8Tuning for matrix M at `batch` vectors (cached)."""
    if candidates is None:
        candidates = candidates_for(batch, SINGLE_CANDIDATES)
    k = key(M, batch)
    with _lock:
        db = _load()
    if not force and k in db:
        return Q8Tuning(*db[k]["tuning"]), db[k]
    R = int(min(48, max(2, -(-2 * L2_BYTES // max(1, M.payload_bytes)))))
    mats = copies(M, R)
    x = torch.randint(-127, 128, (batch, M.cols), dtype=torch.int8, device=M.device)
    y = torch.empty((batch, M.rows), dtype=torch.int32, device=M.device)
    results = {}
    for cand in candidates:
        t = Q8Tuning(*cand)
        try:
            ms = time_launches([lambda m=m, t=t: m.matvec(x, out=y, tuning=t) for m in mats], reps)
        except _lib.MatvansError:
            continue  # e.g. does not fit shared memory
        results[",".join(map(str, cand))] = 1e3 * ms
    if not results:
        raise RuntimeError("autotune: no candidate launched")
    best = min(results, key=results.get)
    entry = {"tuning": [int(v) for v in best.split(",")], "us": results[best], "all": results, "copies": R}
    _update(k, entry)
    return Q8Tuning(*entry["tuning"]), entry


def stack_key(matrices, batch):
    """Cache key of a stack: GPU, library build, batch and a hash of every job's shape, table mode, segment
    length and size (the order of the jobs is part of it: it is the order of the work queue)."""
    import hashlib
    M0 = matrices[0]
    props = torch.cuda.get_device_properties(M0.device)
    cap = torch.cuda.get_device_capability(M0.device)
    h = hashlib.sha1()
    for M in matrices:
        h.update(f"{M.rows}x{M.cols}|{M.local}|{M.seg_quads}|{M.max_blk_rows}|{M.payload_bytes};".encode())
    return f"{props.name}|sm{cap[0]}{cap[1]}|{_build_id()}|stack{len(matrices)}:{h.hexdigest()[:16]}|B{batch}"


def tune_stack(make_stack, candidates=CANDIDATES, reps=10, key=None, force=False):
    """Best tuning for a Q8Stack built by make_stack(tuning); returns (tuning, {cand: us per launch}).  With a
    key (stack_key), a cached result is reused and a new one stored in the same cache as single matrices."""
    if key is not None and not force:
        with _lock:
            db = _load()
        if key in db:
            return tuple(db[key]["tuning"]), db[key]["all"]
    results = {}
    for cand in candidates:
        try:
            S = make_stack(cand)
            ms = time_launches([S.run], reps)
        except _lib.MatvansError:
            continue
        results[",".join(map(str, cand))] = 1e3 * ms
    best = min(results, key=results.get)
    tuning = tuple(int(v) for v in best.split(","))
    if key is not None:
        _update(key, {"tuning": list(tuning), "us": results[best], "all": results})
    return tuning, results
