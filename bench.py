#!/usr/bin/env python
"""Headline benchmark: entropy-coded int8 matvec on B200.

Metric: int8-equivalent GB/s ((rows*cols + B*cols + 4*B*rows) bytes per matvec
/ time) and us per matvec, with bit-exact int32 output, against the dense int8
dp4a matvec on the same GPU.

Workload (one step): the single-vector 7B-layer shapes W_q 4096x4096,
11008x4096 and 4096x11008, each at sigma 4 and sigma 2
(clamp(round(N(0, sigma^2)))), each encoded once with one global table and once
with per-row tables, in this library's Q8-stripe layout: 12 matvecs with one
int8 x each (B = 1).  All 12 compressed matrices together are ~200 MB, larger
than the 126 MB L2, and each is read once per step, so every read comes from
HBM.  Inputs are synthetic and seeded; there is no public dataset.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's CPU implementation of the path (the
oracle's C restatement of the ans-warp-rows decoder, buffered/
ans-warp-rows-kernel.cu, with all host threads) on the same shapes.
"""
import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPES = [(4096, 4096), (11008, 4096), (4096, 11008)]
SIGMAS = [4.0, 2.0]
METRIC = "us/matvec & int8-equiv GB/s vs dense dp4a int8 on B200, bit-exact int32 output"
UNIT = "GB/s"
L2_BYTES = 126 * 2 ** 20
# DRAM traffic of one launch of the step's kernel, as the latest committed ncu summary of it records
PROFILE_RECORD = os.path.join(ROOT, "profiles", "q8s_kernel_stack12_b1.json")


def profiled_traffic():
    """(dram__bytes_read.sum + dram__bytes_write.sum per launch, source) from the committed profile record, or
    (None, reason) when there is none."""
    try:
        with open(PROFILE_RECORD) as f:
            rec = json.load(f)
        return float(rec["dram_bytes_per_launch"]), f"{os.path.relpath(PROFILE_RECORD, ROOT)}: {rec['command']}"
    except (OSError, ValueError, KeyError):
        return None, "no profile record"


def gen_matrix(shape, sigma, seed):
    rng = np.random.default_rng(seed)
    out = np.empty(shape, np.int8)
    step = max(1, (1 << 24) // shape[1])
    for r0 in range(0, shape[0], step):
        z = rng.standard_normal((min(step, shape[0] - r0), shape[1]), dtype=np.float32) * np.float32(sigma)
        out[r0:r0 + z.shape[0]] = np.clip(np.rint(z), -127, 127).astype(np.int8)
    return out


def workload(seed=20251203):
    mats = []
    for i, shape in enumerate(SHAPES):
        for j, s in enumerate(SIGMAS):
            mats.append(dict(shape=shape, sigma=s, W=gen_matrix(shape, s, seed + 10 * i + j)))
    return mats


def int8_equiv_bytes(rows, cols, B=1):
    return rows * cols + B * cols + 4 * B * rows


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons through NVML while running."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown", 0x1: "gpu_idle"}

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            self.sample()
            time.sleep(0.005)

    def sample(self):
        if not self.nv:
            return
        try:
            self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            for bit, name in self.REASONS.items():
                if r & bit and name != "gpu_idle":
                    self.reasons.add(name)
        except Exception:
            pass

    def __enter__(self):
        self.sample()
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self.t.join()
        self.sample()

    def summary(self):
        return {"sm_mhz": float(np.median(self.samples)) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ------------------------------------------------------------------ CPU legs

def headline_config():
    """The workload both arms measure (the reference arm decodes the same 12 matvecs)."""
    return {"workload": "7B-layer single-vector int8 matvecs: W_q 4096x4096, 11008x4096 and 4096x11008 at sigma 4 "
                        "and 2, each once as a global-CDF and once as a per-row-CDF matvec (12 matvecs per step), "
                        "B=1, seeded synthetic int8 weights and x",
            "batch": 1, "matvecs_per_step": 2 * len(SHAPES) * len(SIGMAS), "seed": 20251203,
            "l2": "inputs larger than L2: the 12 matrices' compressed streams (about 200 MB) exceed the 126 MiB "
                  "L2 and each is read once per step"}


def cpu_encode_all(mats):
    """Each matrix in the reference's ans-warp-rows layout, encoded by the oracle's restatement of the reference
    encoder (buffered/encoder.py:271-470; byte-identical on the reference-made fixtures), so that the CPU legs
    load no product code."""
    import oracle
    out = []
    for m in mats:
        comp, offs, p, c, pr = oracle.awr_encode(m["W"])
        out.append(dict(shape=m["shape"], sigma=m["sigma"], compressed=comp, offsets=offs, ppf=p, cum=c, prob=pr))
    return out


def cpu_reference_pass(awr_mats, x_by_cols, nthreads):
    """One pass of the reference algorithm over the 12 matvecs of a step: the reference has one layout (a global
    CDF per matrix), so each matrix is decoded for its global-CDF and for its per-row-CDF matvec.  Decode + int8
    dot products by the oracle's C restatement of buffered/ans-warp-rows-kernel.cu:20-210."""
    import oracle
    nbytes = 0
    for m in awr_mats:
        rows, cols = m["shape"]
        for _ in range(2):
            y = oracle.awr_matvec(m["compressed"], m["offsets"], rows, cols, m["ppf"], m["cum"], m["prob"],
                                  x_by_cols[cols], nthreads=nthreads)
            assert y.shape == (rows,)
            nbytes += int8_equiv_bytes(rows, cols)
    return nbytes


def cpu_baseline(mats, x_by_cols, budget_s=8.0):
    nthreads = os.cpu_count() or 1
    awr = cpu_encode_all(mats)
    t0 = time.perf_counter()
    nbytes, passes = 0, 0
    while True:
        nbytes += cpu_reference_pass(awr, x_by_cols, nthreads)
        passes += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": nbytes / dt / 1e9, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{passes} pass(es) over the step's 12 matvecs (the 6 matrices in the reference's "
                      f"ans-warp-rows layout, each decoded twice), oracle C decode+matvec, {nthreads} threads, "
                      f"{dt:.1f} s"}


def run_reference(args):
    """The reference's CPU implementation of the path on this host's cores: no product library is loaded."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    mats = workload()
    rng = np.random.default_rng(7)
    x_by_cols = {c: rng.integers(-127, 128, size=c).astype(np.int8) for c in {s[1] for s in SHAPES}}
    awr = cpu_encode_all(mats)
    nthreads = os.cpu_count() or 1
    # gate: every decoded product equals the int64 matvec of the original matrix
    import oracle
    for m, a in zip(mats, awr):
        rows, cols = m["shape"]
        y = oracle.awr_matvec(a["compressed"], a["offsets"], rows, cols, a["ppf"], a["cum"], a["prob"],
                              x_by_cols[cols], nthreads=nthreads)
        if not np.array_equal(y, oracle.matvec_i8(m["W"], x_by_cols[cols])):
            raise SystemExit("bench --impl reference: decoded product is not exact")
    for _ in range(args.warmup):
        cpu_reference_pass(awr, x_by_cols, nthreads)
    t0 = time.perf_counter()
    nbytes = 0
    for _ in range(args.steps):
        nbytes += cpu_reference_pass(awr, x_by_cols, nthreads)
    dt = time.perf_counter() - t0
    value = nbytes / dt / 1e9
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8", "data": "synthetic",
            "impl": "reference", "config": headline_config(),
            "layout": "the reference's ans-warp-rows layout (one global CDF per matrix, its only layout), encoded by "
                      "the oracle's restatement of buffered/encoder.py",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"each step one pass over the 12 matvecs with the oracle's C restatement of "
                                       f"the reference decoder (buffered/ans-warp-rows-kernel.cu), {nthreads} "
                                       f"threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ batched stack (224 matrices)

LAYER = [("q", 4096, 4096), ("k", 4096, 4096), ("v", 4096, 4096), ("o", 4096, 4096),
         ("gate", 11008, 4096), ("up", 11008, 4096), ("down", 4096, 11008)]


def stack_specs(layers=32, seed=20251204):
    """7 matrices per layer; each with its own sigma ~ U[2,6]; 10% of them
    Laplace(b=3) with 0.1% outliers at +-100 instead."""
    rng = np.random.default_rng(seed)
    n = layers * len(LAYER)
    lap = set(rng.choice(n, size=int(round(0.1 * n)), replace=False).tolist())
    specs = []
    for i in range(n):
        name, r, c = LAYER[i % len(LAYER)]
        specs.append(dict(name=f"L{i // len(LAYER)}.{name}", rows=r, cols=c, sigma=float(rng.uniform(2, 6)),
                          laplace=i in lap, seed=seed + 1 + i))
    return specs


def gen_on_device(torch, spec, dev):
    """Seeded int8 weights generated on the GPU (host numpy generation of 6.5 G weights takes minutes)."""
    g = torch.Generator(device=dev)
    g.manual_seed(spec["seed"])
    shape = (spec["rows"], spec["cols"])
    if spec["laplace"]:
        e1 = torch.empty(shape, device=dev).exponential_(generator=g)
        e2 = torch.empty(shape, device=dev).exponential_(generator=g)
        z = 3.0 * (e1 - e2)
        del e1, e2
        u = torch.rand(shape, device=dev, generator=g)
        z = torch.where(u < 0.0005, torch.full_like(z, -100.0), torch.where(u < 0.001, torch.full_like(z, 100.0), z))
        del u
    else:
        z = torch.randn(shape, device=dev, generator=g) * spec["sigma"]
    return torch.clamp(torch.round(z), -127, 127).to(torch.int8)


def entropy_dev(torch, Wd):
    cnt = torch.bincount((Wd.reshape(-1).to(torch.int32) + 128), minlength=256).double()
    p = cnt[cnt > 0] / cnt.sum()
    return float(-(p * torch.log2(p)).sum())


def build_stack(torch, ops, dev, layers=32, keep_dense=True):
    from matvans_b200 import codec
    mats = []
    for sp in stack_specs(layers):
        Wd = gen_on_device(torch, sp, dev)
        M = ops.Q8Matrix(codec.q8_encode(Wd.cpu().numpy(), local=True), dev)
        mats.append(dict(spec=sp, M=M, Wd=Wd if keep_dense else None, entropy=entropy_dev(torch, Wd)))
    return mats


def chain_section(torch, ops, autotune, dev, mats, batches=(1, 16), reps=5, scale=2e-3):
    """The reference's chained workload over the stack's q,k,v,o,gate,down matrices (192, 4096 -> 4096 ->
    ... -> 11008 -> 4096 per layer): x_{j+1} = clamp(rn(fp32(W_j x_j) * scale)).  Fused (one cooperative
    launch), one chain launch per matrix, and the same matrices as an independent stack (no dependencies).
    Gate: every step against the dense kernel and torch's fp32 round-half-even on the GPU."""
    chain = [m for m in mats if not m["spec"]["name"].endswith(".up")]
    Ms = [m["M"] for m in chain]
    out = {"matrices": len(Ms)}
    g = torch.Generator(device=dev)
    g.manual_seed(123)
    for B in batches:
        x0 = torch.randint(-127, 128, (B, Ms[0].cols), dtype=torch.int8, device=dev, generator=g)
        C = ops.Q8Chain(Ms, [scale] * len(Ms), batch=B, x0=x0, device=dev)
        C.run()
        torch.cuda.synchronize()
        v = x0
        for j, m in enumerate(chain):
            y = ops.dense_matvec(m["Wd"], v)
            v = torch.clamp(torch.round(y.float() * scale), -128, 127).to(torch.int8)
            got = C.xs[j + 1] if j + 1 < len(Ms) else C.out8
            if not torch.equal(got, v):
                raise SystemExit(f"bench: chain step {j} (B={B}) is not bit-exact")
        t_fused, gf = time_graph(torch, C.run, reps)
        del gf
        steps, xin = [], x0
        for M in Ms:
            c = ops.Q8Chain([M], [scale], batch=B, x0=xin, device=dev)
            steps.append(c)
            xin = c.out8
        t_each, ge = time_graph(torch, lambda: [c.run() for c in steps], reps)
        del ge
        S = ops.Q8Stack(Ms, batch=B, device=dev)
        t_stack, gs = time_graph(torch, S.run, reps)
        del gs, S, steps
        out[f"B{B}"] = {"fused_us": round(1e3 * t_fused, 1), "one_launch_per_matrix_us": round(1e3 * t_each, 1),
                        "independent_stack_us": round(1e3 * t_stack, 1),
                        "fused_speedup_vs_per_matrix": round(t_each / t_fused, 3)}
    return out


def stack_section(torch, ops, autotune, dev, batches=(1, 4, 8, 16), layers=32, reps=10):
    """The 224-matrix uneven stack, one persistent launch per step, B in {1,4,8,16}; the tensor-core
    engine competes with dp4a from 3 vectors on.  Gate: bit-exact against the dense int8 kernel on the same x."""
    t_build = time.perf_counter()
    mats = build_stack(torch, ops, dev, layers)
    t_build = time.perf_counter() - t_build
    Ms = [m["M"] for m in mats]
    weights = sum(M.rows * M.cols for M in Ms)
    comp = sum(M.payload_bytes for M in Ms)
    out = {"matrices": len(Ms), "weights": weights, "compressed_bytes": comp,
           "bits_per_weight": 8.0 * comp / weights,
           "entropy_bits_mean": float(np.mean([m["entropy"] for m in mats])),
           "laplace_matrices": sum(m["spec"]["laplace"] for m in mats), "build_s": round(t_build, 1), "batches": {}}
    g = torch.Generator(device=dev)
    g.manual_seed(99)
    for B in batches:
        xs = [torch.randint(-127, 128, (B, M.cols), dtype=torch.int8, device=dev, generator=g) for M in Ms]
        ref = [torch.empty((B, M.rows), dtype=torch.int32, device=dev) for M in Ms]

        def dense_step():
            for m, x, y in zip(mats, xs, ref):
                ops.dense_matvec(m["Wd"], x, out=y)

        t_dense, gd = time_graph(torch, dense_step, reps)
        del gd
        t_gemm = None
        if B % 8 == 0:
            xts = [x.t() for x in xs]
            t_gemm, gg = time_graph(torch, lambda: [torch._int_mm(m["Wd"], xt) for m, xt in zip(mats, xts)], reps)
            del gg
            for m, xt, yr in zip(mats, xts, ref):
                if not torch.equal(torch._int_mm(m["Wd"], xt).t(), yr):
                    raise SystemExit(f"bench: cuBLAS int8 GEMM disagrees with dense dp4a on {m['spec']['name']}")
        cands = autotune.candidates_for(B, autotune.CANDIDATES)
        best, res = autotune.tune_stack(lambda t: ops.Q8Stack(Ms, batch=B, tuning=t, xs=xs, device=dev),
                                        candidates=cands, reps=reps, key=autotune.stack_key(Ms, B))
        row = {}
        # tensor cores: engine 0; CUDA cores: engine 1 (0 below the tensor cores' smallest batch)
        groups = {"tcgen05": (0,), "dp4a": (1,)} if B >= ops.MMA_MIN_BATCH else {"dp4a": (0,)}
        for name, engs in groups.items():
            mine = {k: v for k, v in res.items() if int(k.split(",")[5]) in engs}
            if not mine:
                continue
            kbest = min(mine, key=mine.get)
            S = ops.Q8Stack(Ms, batch=B, tuning=tuple(int(v) for v in kbest.split(",")), xs=xs, device=dev)
            S.run()
            torch.cuda.synchronize()
            for y, yr, m in zip(S.ys, ref, mats):
                if not torch.equal(y, yr):
                    raise SystemExit(f"bench: stack {m['spec']['name']} B={B} tuning {kbest} is not bit-exact")
            t_ms, gs = time_graph(torch, S.run, reps)
            del gs, S
            row[name] = {"us_per_step": round(1e3 * t_ms, 1), "tuning": kbest,
                         "int8_equiv_gbs": round(sum(int8_equiv_bytes(M.rows, M.cols, B) for M in Ms) / t_ms / 1e6, 1),
                         "compressed_gbs": round(comp / t_ms / 1e6, 1),
                         "us_per_matvec": round(1e3 * t_ms / len(Ms), 3)}
        fastest = min(row.values(), key=lambda v: v["us_per_step"])
        row["candidates_us"] = {k: round(v, 1) for k, v in sorted(res.items(), key=lambda kv: kv[1])}
        row["dense_dp4a_us_per_step"] = round(1e3 * t_dense, 1)
        row["speedup_vs_dense_dp4a"] = round(1e3 * t_dense / fastest["us_per_step"], 3)
        row["cublas_int8_gemm_us_per_step"] = None if t_gemm is None else round(1e3 * t_gemm, 1)
        row["speedup_vs_cublas_int8_gemm"] = None if t_gemm is None else round(1e3 * t_gemm / fastest["us_per_step"], 3)
        # the faster of the two dense baselines (dp4a, and cuBLAS int8 GEMM where its shape rules allow it)
        row["speedup_vs_best_dense"] = round(1e3 * min(t_dense, t_gemm or 1e30) / fastest["us_per_step"], 3)
        out["batches"][f"B{B}"] = row
        del xs, ref
    out["chain192"] = chain_section(torch, ops, autotune, dev, mats, reps=reps)
    del mats, Ms
    torch.cuda.empty_cache()
    ops.device_status()
    return out


# ------------------------------------------------------------------ large low-entropy matrices

LARGE_SHAPES = [(16384, 16384), (28672, 8192)]
LARGE_DISTS = [("laplace_b2", None), ("normal_s1", 1.0)]


def gen_large(torch, shape, dist, seed, dev):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    if dist == "laplace_b2":
        z = 2.0 * (torch.empty(shape, device=dev).exponential_(generator=g) -
                   torch.empty(shape, device=dev).exponential_(generator=g))
    else:
        z = torch.randn(shape, device=dev, generator=g)
    return torch.clamp(torch.round(z), -127, 127).to(torch.int8)


def int8_gemm_us(torch, Ws, x, reps=10):
    """cuBLAS int8 tensor-core GEMM (torch._int_mm, exact int32) y^T = W x^T over rotating copies of W, in us
    per matrix; None where its shape rules (> 16 rows, columns and vectors in multiples of 8) exclude it."""
    B, cols = x.shape
    if B % 8 or cols % 8 or Ws[0].shape[0] <= 16:
        return None
    xt = x.t()  # [cols, B], column-major
    try:
        t, _ = time_graph(torch, lambda: [torch._int_mm(w, xt) for w in Ws], reps, inner=len(Ws))
    except RuntimeError:
        return None
    return 1e3 * t


def large_section(torch, ops, autotune, dev, batches=(1, 16)):
    """Large low-entropy matrices: 16384x16384 and 28672x8192, Laplace(b=2) and round(N(0,1)), per-row tables, B in {1, 16}:
    us per matvec of the autotuned single launch and of dense dp4a, bits/weight vs entropy, HBM GB/s."""
    from matvans_b200 import codec
    out = {}
    gen = torch.Generator(device=dev)
    gen.manual_seed(5)
    for i, shape in enumerate(LARGE_SHAPES):
        for j, (dist, _) in enumerate(LARGE_DISTS):
            Wd = gen_large(torch, shape, dist, 4000 + 10 * i + j, dev)
            M = ops.Q8Matrix(codec.q8_encode(Wd.cpu().numpy(), local=True), dev)
            rows, cols = shape
            row = {"bits_per_weight": round(M.bits_per_weight, 3), "entropy_bits": round(entropy_dev(torch, Wd), 3),
                   "compressed_bytes": M.payload_bytes}
            Ws = [Wd] + [Wd.clone() for _ in range(copies_for(rows * cols) - 1)]
            for B in batches:
                x = torch.randint(-127, 128, (B, cols), dtype=torch.int8, device=dev, generator=gen)
                yd = torch.empty((B, rows), dtype=torch.int32, device=dev)
                t_dense, _ = time_graph(torch, lambda: [ops.dense_matvec(w, x, out=yd) for w in Ws], 10, inner=len(Ws))
                tun, _ = autotune.tune(M, batch=B)
                y = M.matvec(x, tuning=tun)
                ops.dense_matvec(Wd, x, out=yd)
                torch.cuda.synchronize()
                if not torch.equal(y, yd):
                    raise SystemExit(f"bench: large {shape} {dist} B={B} is not bit-exact")
                # the launch shape may come from the cache; the time is taken here, on rotating copies (cold L2)
                Ms = autotune.copies(M, copies_for(M.payload_bytes))
                yq = torch.empty((B, rows), dtype=torch.int32, device=dev)
                us = 1e3 * time_graph_med(torch, lambda: [Mi.matvec(x, out=yq, tuning=tun) for Mi in Ms], 10,
                                          inner=len(Ms))
                del Ms
                alg = M.payload_bytes + B * cols + 4 * B * rows
                gemm = int8_gemm_us(torch, Ws, x)
                if gemm is not None:
                    ref = torch._int_mm(Wd, x.t()).t()
                    if not torch.equal(ref, yd):
                        raise SystemExit(f"bench: cuBLAS int8 GEMM disagrees with dense dp4a on {shape} {dist}")
                row[f"B{B}"] = {"us": round(us, 2), "dense_dp4a_us": round(1e3 * t_dense, 2),
                                "speedup_vs_dense_dp4a": round(1e3 * t_dense / us, 3),
                                "cublas_int8_gemm_us": None if gemm is None else round(gemm, 2),
                                "speedup_vs_cublas_int8_gemm": None if gemm is None else round(gemm / us, 3),
                                "speedup_vs_best_dense": round(min(1e3 * t_dense, gemm or 1e30) / us, 3),
                                "int8_equiv_gbs": round(int8_equiv_bytes(rows, cols, B) / us / 1e3, 1),
                                "compressed_gbs": round(alg / us / 1e3, 1),
                                "tuning": [tun.warps, tun.ilp, tun.depth, tun.ctas_per_sm, tun.parts, tun.engine]}
            out[f"{rows}x{cols}_{dist}"] = row
            del Ws, Wd, M
            torch.cuda.empty_cache()
    ops.device_status()
    return out


# ------------------------------------------------------------------ the reference's own CUDA kernels

def _ref_libs():
    """ctypes handles of the reference kernels built by oracle/build_ref.py (bench comparators), or {}."""
    import ctypes
    d = os.path.join(ROOT, "oracle", "_ref")
    out = {}
    for key, fn in (("awr", "libref_awr.so"), ("dense", "libref_dense.so"), ("wpr", "libref_wpr.so"),
                    ("wpr_local", "libref_wpr_local.so")):
        path = os.path.join(d, fn)
        if os.path.exists(path):
            out[key] = ctypes.CDLL(path)
    return out


def reference_kernels_section(torch, ops, dev, mats, xd, ours_us):
    """The reference's own kernels (compiled unmodified for sm_100a by oracle/build_ref.py) on the sigma-4
    matrices of the workload, each launched with the reference's own launch shape over rotating copies (cold
    L2), next to this library's kernels on the same matrices.  Every stream buffer is padded so that the
    kernels' known over-reads past a row's end stay inside it.  Gates: dense and WPR int32 y exact; AWR's
    int8 output equal to clamp(rn(fp32(y) * scale))."""
    import ctypes
    libs = _ref_libs()
    if not libs:
        return {"unavailable": "oracle/_ref was not built (the reference checkout was absent at build time)"}
    P = ctypes.c_void_p
    stream = lambda: P(torch.cuda.current_stream().cuda_stream)  # noqa: E731
    out = {}
    for m in mats:
        if m["sigma"] != 4.0:
            continue
        rows, cols = m["shape"]
        key = f"{rows}x{cols}"
        row = {}
        W = m["W"]
        x1 = xd[cols]
        y_exact = (W.astype(np.int32) @ x1.cpu().numpy().astype(np.int32)).astype(np.int32)
        if "dense" in libs:
            L = libs["dense"]
            Wd = torch.from_numpy(W).to(dev)
            Ws = [Wd] + [Wd.clone() for _ in range(copies_for(rows * cols) - 1)]
            yd = torch.empty(rows, dtype=torch.int32, device=dev)
            run = lambda w: L.ref_dense_launch(P(yd.data_ptr()), P(w.data_ptr()), P(x1.data_ptr()), cols, rows,  # noqa
                                               stream())
            if run(Wd) != 0:
                row["dense_dp4a"] = "launch failed"
            else:
                torch.cuda.synchronize()
                if not np.array_equal(yd.cpu().numpy(), y_exact):
                    row["dense_dp4a"] = "output differs from the exact product"
                else:
                    t = time_graph_med(torch, lambda: [run(w) for w in Ws], 10, inner=len(Ws))
                    row["dense_dp4a_us"] = round(1e3 * t, 2)
            del Ws, Wd
        if "awr" in libs:
            L = libs["awr"]
            A = ops.AwrMatrix.encode(W, device=dev)
            pad = 1024  # words past the stream: a row's last refill reads 32 uint4 ahead

            def padded():
                c = torch.zeros(A.n_words + pad, dtype=torch.int32, device=dev)
                c[:A.n_words].copy_(A.compressed.view(torch.int32))
                return c
            comps = [padded() for _ in range(copies_for(4 * A.n_words))]
            out8 = torch.empty(rows, dtype=torch.int8, device=dev)
            scale = np.float32(127.0) / np.float32(max(1, int(np.abs(y_exact).max())))
            run = lambda c: L.ref_awr_launch(P(out8.data_ptr()), P(c.data_ptr()), P(A.offsets.data_ptr()),  # noqa
                                             P(A.ppf.data_ptr()), P(A.ppf_cum.data_ptr()), P(A.ppf_prob.data_ptr()),
                                             P(x1.data_ptr()), cols, rows, ctypes.c_float(float(scale)), stream())
            if run(comps[0]) != 0:
                row["ans_warp_rows"] = "launch failed"
            else:
                torch.cuda.synchronize()
                ref8 = np.clip(np.rint(y_exact.astype(np.float32) * scale), -128, 127).astype(np.int8)
                if not np.array_equal(out8.cpu().numpy(), ref8):
                    row["ans_warp_rows"] = "output differs from clamp(rn(y * scale))"
                else:
                    t = time_graph_med(torch, lambda: [run(c) for c in comps], 5, inner=len(comps))
                    row["ans_warp_rows_us"] = round(1e3 * t, 2)
            del comps, A
        if rows == cols and cols % 512 == 0 and cols <= 4096 and ("wpr" in libs or "wpr_local" in libs):
            Pm = ops.WprMatrix.encode(W, device=dev)

            def padded_payload():
                c = torch.zeros(Pm.payload_size + 4096, dtype=torch.int16, device=dev)
                c[:Pm.payload_size].copy_(Pm.payload[:Pm.payload_size].view(torch.int16))
                return c
            pays = [padded_payload() for _ in range(copies_for(2 * Pm.payload_size))]
            yw = torch.empty(rows, dtype=torch.int32, device=dev)
            for name in ("wpr", "wpr_local"):
                if name not in libs:
                    continue
                L = libs[name]
                run = lambda p, L=L: L.ref_wpr_launch(  # noqa: E731
                    P(yw.data_ptr()), P(x1.data_ptr()), rows, cols, P(Pm.cursors.data_ptr()),
                    ctypes.c_int8(Pm.min_value), ctypes.c_uint8(Pm.G), P(Pm.cdf.data_ptr()), P(Pm.ppf.data_ptr()),
                    P(p.data_ptr()), Pm.payload_size, stream())
                label = "matvansWarpPerRow" if name == "wpr" else "matvansWarpPerRow_local_cdf"
                if run(pays[0]) != 0:
                    row[label] = "launch failed"
                    continue
                torch.cuda.synchronize()
                if not np.array_equal(yw.cpu().numpy(), y_exact):
                    row[label] = "output differs from the exact product"
                    continue
                t = time_graph_med(torch, lambda: [run(p) for p in pays], 5, inner=len(pays))
                row[label + "_us"] = round(1e3 * t, 2)
            del pays, Pm
        for k, v in ours_us.items():
            if k.startswith(key + "_s4_"):
                row[f"ours_{k.split('_')[-1]}_us"] = round(v, 2)
        best = min((v for k, v in ours_us.items() if k.startswith(key + "_s4_")), default=None)
        if best:
            for k in ("dense_dp4a_us", "ans_warp_rows_us", "matvansWarpPerRow_us", "matvansWarpPerRow_local_cdf_us"):
                if k in row:
                    row["speedup_vs_" + k[:-3]] = round(row[k] / best, 3)
        out[key] = row
        torch.cuda.empty_cache()
    ops.device_status()
    return out


# ------------------------------------------------------------------ GPU arm

def time_graph(torch, fn, reps, inner=1):
    """Capture fn() into a graph, replay `reps` times; returns ms per fn() call."""
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        fn()
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps / inner, g


def time_graph_med(torch, fn, reps, inner=1, windows=10):
    """Like time_graph, but the median over `windows` windows of `reps` replays (ms per fn() call / inner)."""
    _, g = time_graph(torch, fn, 1, inner)
    ts = []
    for _ in range(windows):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            g.replay()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / reps / inner)
    del g
    return float(np.median(ts))


def copies_for(nbytes):
    return int(min(64, max(2, -(-2 * L2_BYTES // max(1, nbytes)))))


def run_ours(args):
    import torch
    from matvans_b200 import dist as mvd

    rank, world, local = mvd.env_rank()
    torch.cuda.set_device(local)
    # rank 0 runs the comparator sections (about a minute) while the others wait at the final barrier
    mvd.init("nccl", timeout_s=900, device=torch.device("cuda", local))

    from matvans_b200 import codec, ops

    dev = torch.device("cuda", local)
    mats = workload()
    rng = np.random.default_rng(7)
    x_by_cols = {c: rng.integers(-127, 128, size=c).astype(np.int8) for c in {s[1] for s in SHAPES}}
    xd = {c: torch.from_numpy(v).to(dev) for c, v in x_by_cols.items()}

    entries = []
    for m in mats:
        H = codec.entropy_bits(m["W"])
        for local_cdf in (False, True):
            M = ops.Q8Matrix.encode(m["W"], local=local_cdf, device=dev)
            rows, cols = m["shape"]
            entries.append(dict(name=f"{rows}x{cols}_s{int(m['sigma'])}_{'local' if local_cdf else 'global'}",
                                M=M, rows=rows, cols=cols, sigma=m["sigma"], entropy=H, W=m["W"],
                                alg_bytes=M.payload_bytes + cols + 4 * rows))
    xs = [xd[e["cols"]][None].contiguous() for e in entries]

    # one step = one persistent launch over all 12 matrices (mv_q8_stack_matvec)
    from matvans_b200 import autotune
    if args.tuning:
        stack_tuning, stack_cands = tuple(int(v) for v in args.tuning.split(",")), {}
    else:
        stack_tuning, stack_cands = autotune.tune_stack(
            lambda t: ops.Q8Stack([e["M"] for e in entries], batch=1, tuning=t, xs=xs, device=dev),
            key=autotune.stack_key([e["M"] for e in entries], 1))
    S = ops.Q8Stack([e["M"] for e in entries], batch=1, tuning=stack_tuning, xs=xs, device=dev)
    # correctness gate before timing: bit-exact against the host int64 matvec
    S.run()
    for e, y in zip(entries, S.ys):
        ref = (e["W"].astype(np.int32) @ x_by_cols[e["cols"]].astype(np.int32))
        if not np.array_equal(y.cpu().numpy()[0], ref):
            raise SystemExit(f"bench: {e['name']} is not bit-exact")
    ops.device_status()

    def step():
        S.run()

    if args.profile:  # small fixed case for ncu: the gate above + two plain steps
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        ops.device_status()
        mvd.shutdown()
        return 0

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    _, g = time_graph(torch, step, 3)
    for _ in range(max(args.warmup, 3)):
        g.replay()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    # exactly K steps between a barrier + synchronize on both sides, recorded in >= 10 windows; the step
    # time is the median window (per-window means), and the job's time the slowest rank's
    nwin = max(1, min(10, args.steps))
    bounds = [round(i * args.steps / nwin) for i in range(nwin + 1)]
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(nwin + 1)]
    mvd.barrier()
    torch.cuda.synchronize()
    with sampler:
        evs[0].record()
        for w in range(nwin):
            for _ in range(bounds[w + 1] - bounds[w]):
                g.replay()
            evs[w + 1].record()
        torch.cuda.synchronize()
    mvd.barrier()
    win_ms = [evs[w].elapsed_time(evs[w + 1]) / max(1, bounds[w + 1] - bounds[w]) for w in range(nwin)]
    step_bytes = sum(int8_equiv_bytes(e["rows"], e["cols"]) for e in entries)
    value, sec = mvd.aggregate_throughput(step_bytes / 1e9, float(np.median(win_ms)) * 1e-3, device=dev)
    ms = sec * 1e3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    alg = sum(e["alg_bytes"] for e in entries)
    peak, peak_kind = measured_peak()
    achieved = alg / (ms * 1e-3) / 1e9
    ops.device_status()

    # end to end through the public API: pinned host x in, int32 y out, every step.  The distinct x
    # vectors sit in one pinned buffer (one host-to-device copy into one device buffer that the jobs' x
    # are views of) and the stack's outputs are views of its y_flat (one device-to-host copy).  Two such
    # pipelines alternate, as a serving loop would run them: step k's output copy (on a copy stream)
    # overlaps step k + 1's input copy and decode, and a pipeline's buffers are reused only after its
    # previous output copy has finished; the next step's input copy (a third stream) overlaps the decode too.
    cols_list = sorted(x_by_cols)
    xh_flat = torch.from_numpy(np.concatenate([x_by_cols[c] for c in cols_list])).pin_memory()
    offs = np.cumsum([0] + cols_list)
    pipes = []
    for _ in range(2):
        x_dev_flat = torch.empty_like(xh_flat, device=dev)
        xin = {c: x_dev_flat[offs[i]:offs[i + 1]].view(1, c) for i, c in enumerate(cols_list)}
        S_e2e = ops.Q8Stack([e["M"] for e in entries], batch=1, tuning=stack_tuning,
                            xs=[xin[e["cols"]] for e in entries], device=dev)
        yh_flat = torch.empty(S_e2e.y_flat.numel(), dtype=torch.int32).pin_memory()
        pipes.append(dict(x=x_dev_flat, S=S_e2e, yh=yh_flat, xin=torch.cuda.Event(), ran=torch.cuda.Event(),
                          out=torch.cuda.Event()))
    comp = torch.cuda.current_stream()
    h2d_stream, copy_stream = torch.cuda.Stream(), torch.cuda.Stream()

    def e2e_step(k):
        P = pipes[k & 1]
        # input copy on its own stream, as soon as this pipeline's previous decode has read x
        h2d_stream.wait_event(P["ran"])
        with torch.cuda.stream(h2d_stream):
            P["x"].copy_(xh_flat, non_blocking=True)
            P["xin"].record(h2d_stream)
        comp.wait_event(P["xin"])
        comp.wait_event(P["out"])  # this pipeline's previous output copy has finished reading y_flat
        P["S"].run()
        P["ran"].record(comp)
        copy_stream.wait_event(P["ran"])
        with torch.cuda.stream(copy_stream):
            P["yh"].copy_(P["S"].y_flat, non_blocking=True)
            P["out"].record(copy_stream)

    for k in range(4):
        e2e_step(k)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record()
    for k in range(args.steps):
        e2e_step(k)
    comp.wait_stream(copy_stream)  # the last output copy is inside the timed region
    comp.wait_stream(h2d_stream)
    e1.record()
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / args.steps * 1e3
    # the slowest rank sets the job's time, as for the device-timed value
    e2e_ms = mvd.max_over_ranks(max(e0.elapsed_time(e1) / args.steps, wall), device=dev)
    yh_flat = pipes[(args.steps - 1) & 1]["yh"]
    h2d = xh_flat.numel()
    d2h = 4 * yh_flat.numel()
    # the outputs that came back to the host (both pipelines) are the gated ones
    if not all(torch.equal(P["yh"], S.y_flat.cpu()) for P in pipes):
        raise SystemExit("bench: end-to-end outputs differ from the device-timed step's")

    # comparators and the other configurations: rank 0 only (the others wait at the final barrier)
    extras = rank == 0

    # per-matrix us/matvec with rotating copies (cold L2), and the comparators
    per = {}
    for e in (entries if extras else []):
        M = e["M"]
        tun, _ = autotune.tune(M, batch=1)  # the launch shape may come from the cache; the time is taken here
        Ms = autotune.copies(M, copies_for(M.payload_bytes))
        x1 = xd[e["cols"]][None]
        y1 = torch.empty((1, e["rows"]), dtype=torch.int32, device=dev)
        t_ms = time_graph_med(torch, lambda: [Mi.matvec(x1, out=y1, tuning=tun) for Mi in Ms], 10, inner=len(Ms))
        del Ms
        per[e["name"]] = {"us": 1e3 * t_ms, "int8_equiv_gbs": int8_equiv_bytes(e["rows"], e["cols"]) / t_ms / 1e6,
                          "compressed_gbs": e["alg_bytes"] / t_ms / 1e6, "bits_per_weight": M.bits_per_weight,
                          "entropy_bits": e["entropy"],
                          "tuning": [tun.warps, tun.ilp, tun.depth, tun.ctas_per_sm, tun.parts]}
    torch.cuda.empty_cache()
    dense, cublas, awr_t, wpr_t, aws_t = {}, {}, {}, {}, {}
    for m in (mats if extras else []):
        if m["sigma"] != 4.0:
            continue
        rows, cols = m["shape"]
        key = f"{rows}x{cols}"
        Wd = torch.from_numpy(m["W"]).to(dev)
        R = copies_for(rows * cols)
        Ws = [Wd] + [Wd.clone() for _ in range(R - 1)]
        yd = torch.empty((1, rows), dtype=torch.int32, device=dev)
        x1 = xd[cols][None]
        t_ms, _ = time_graph(torch, lambda: [ops.dense_matvec(w, x1, out=yd) for w in Ws], 20, inner=R)
        dense[key] = {"us": 1e3 * t_ms, "int8_equiv_gbs": int8_equiv_bytes(rows, cols) / t_ms / 1e6}
        del Ws
        Wf = Wd.float()
        R = copies_for(4 * rows * cols)
        Wfs = [Wf] + [Wf.clone() for _ in range(R - 1)]
        xf = xd[cols].float()
        t_ms, _ = time_graph(torch, lambda: [torch.mv(w, xf) for w in Wfs], 20, inner=R)
        cublas[key] = {"us": 1e3 * t_ms}
        del Wfs, Wf, Wd
        A = ops.AwrMatrix.encode(m["W"], device=dev)
        R = copies_for(4 * A.n_words)
        As = [A] + [ops.AwrMatrix(A.compressed.cpu().numpy(), A.offsets.cpu().numpy(), A.ppf.cpu().numpy(),
                                  A.ppf_cum.cpu().numpy(), A.ppf_prob.cpu().numpy(), rows, cols, dev)
                    for _ in range(R - 1)]
        t_ms, _ = time_graph(torch, lambda: [a.matvec(x1, out=yd) for a in As], 10, inner=R)
        awr_t[key] = {"us": 1e3 * t_ms, "bits_per_weight": 32.0 * A.n_words / (rows * cols)}
        del As, A
        S_ = ops.AwsMatrix.encode(m["W"], device=dev)
        R = copies_for(4 * S_.n_words)
        Ss = [S_] + [ops.AwsMatrix(S_.compressed.cpu().numpy(), S_.offsets.cpu().numpy(), S_.ppf.cpu().numpy(),
                                   S_.ppf_cum.cpu().numpy(), S_.ppf_prob.cpu().numpy(), rows, cols, dev)
                     for _ in range(R - 1)]
        t_ms, _ = time_graph(torch, lambda: [a.matvec(x1, out=yd) for a in Ss], 10, inner=R)
        aws_t[key] = {"us": 1e3 * t_ms, "bits_per_weight": 32.0 * S_.n_words / (rows * cols)}
        del Ss, S_
        if cols % 512 == 0 and rows == cols:
            P = ops.WprMatrix.encode(m["W"], device=dev)
            R = copies_for(2 * P.payload_size)
            from matvans_b200.codec import CompressedMatrix
            cm = CompressedMatrix(rows, cols, 1.0, P.cursors.cpu().numpy(), P.min_value, P.cdf.cpu().numpy(),
                                  P.ppf.cpu().numpy(), P.payload.cpu().numpy()[:P.payload_size])
            Ps = [P] + [ops.WprMatrix(cm, dev) for _ in range(R - 1)]
            t_ms, _ = time_graph(torch, lambda: [p.matvec(x1, out=yd) for p in Ps], 10, inner=R)
            wpr_t[key] = {"us": 1e3 * t_ms, "bits_per_weight": 16.0 * P.payload_size / (rows * cols)}
            del Ps, P
        torch.cuda.empty_cache()

    ref_kernels = reference_kernels_section(torch, ops, dev, mats, xd, {k: v["us"] for k, v in per.items()}) \
        if extras else None

    # float form (4096x11008 and 11008x4096, sigma 4, per-row scales): forward and re-decoding backward, us per call
    float_form = {}
    for m in (mats if extras else []):
        if m["sigma"] != 4.0 or m["shape"] == (4096, 4096):
            continue
        rows, cols = m["shape"]
        Mf = [e["M"] for e in entries if e["rows"] == rows and e["cols"] == cols and e["sigma"] == 4.0
              and e["M"].local][0]
        s_f = torch.from_numpy(np.random.default_rng(3).uniform(1e-3, 1e-2, rows).astype(np.float32)).to(dev)
        for B in (1, 8, 64):
            Xb = torch.randn((B, cols), device=dev).to(torch.bfloat16)
            dYb = torch.randn((B, rows), device=dev).to(torch.bfloat16)
            yf = torch.empty((B, rows), dtype=torch.float32, device=dev)
            dxf = torch.empty((B, cols), dtype=torch.float32, device=dev)
            tf, _ = time_graph(torch, lambda: Mf.matvec_bf16(Xb, s_f, out=yf), 10)
            tb, _ = time_graph(torch, lambda: Mf.matvec_t_bf16(dYb, s_f, out=dxf), 10)
            float_form[f"{rows}x{cols}_B{B}"] = {"fwd_us": 1e3 * tf, "bwd_us": 1e3 * tb, "bwd_over_fwd": tb / tf}
    ops.device_status()

    stack224 = None if (args.no_stack or not extras) else stack_section(torch, ops, autotune, dev)
    large = None if (args.no_stack or not extras) else large_section(torch, ops, autotune, dev)


    traffic, traffic_src = profiled_traffic()
    line = None
    if rank == 0:
        cb = None
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline(mats, x_by_cols)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8", "data": "synthetic",
            "config": headline_config(),
            "layout": "Q8-stripe layout: 6 matrices with one global table, 6 with per-row tables; working set "
                      f"{alg / 2**20:.0f} MiB of compressed streams, tables and offsets",
            "timing": "CUDA graph of one step (one persistent launch over the 12 matrices), CUDA events over K "
                      "replays in windows, max over ranks; ms_per_step is the median window",
            "stack_tuning": list(stack_tuning), "stack_candidates_us": stack_cands,
            "us_per_matvec": {k: round(v["us"], 3) for k, v in per.items()},
            "per_matrix": per,
            "reference_kernels": ref_kernels,
            "step_windows_ms": [round(v, 4) for v in win_ms],
            "dense_dp4a": dense, "cublas_sgemv_fp32": cublas, "ans_warp_rows_kernel": awr_t,
            "warp_per_row_kernel": wpr_t,
            "ans_warp_stripes_kernel": aws_t,
            "float_form": float_form,
            "stack224": stack224,
            "large_low_entropy": large,
            "speedup_vs_dense_dp4a": {k: round(dense[k.split("_s")[0]]["us"] / v["us"], 3)
                                      for k, v in per.items() if k.split("_s")[0] in dense and "_s4_" in k},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_unit": "bytes per launch",
                         "traffic_source": traffic_src,
                         "algorithmic_bytes": alg, "peak_kind": peak_kind,
                         "kernel": "q8s_kernel<1,ILP,DEPTH> (mv_q8_stack_matvec)",
                         "note": "algorithmic bytes = compressed streams + tables + offsets + x + int32 y"},
            "gpu_launches": args.steps * S.launches_per_run,
            "clocks": sampler.summary(),
            "e2e": {"value": world * step_bytes / (e2e_ms * 1e-3) / 1e9, "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "cpu_baseline": cb,
        }
    del g
    mvd.barrier()
    mvd.shutdown()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def run_profile_kernel(args):
    """Small fixed case of one kernel family for ncu: a bit-exact (or FP64-checked) gate, then two plain
    launches of each kernel.  awr / wpr: 4096x4096 sigma 4, B = 1; dense: 16384x8192 (134 MB, larger than
    L2), B = 1 and B = 16;
    float: 11008x4096 sigma 4, per-row tables, B = 64 forward and backward on the tensor cores."""
    import torch
    from matvans_b200 import ops
    import oracle
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(11)
    if args.profile_kernel in ("float1", "chain", "stripes", "fallback"):
        return run_profile_more(args, torch, ops, oracle, dev, rng)
    if args.profile_kernel == "float":
        shape = (11008, 4096)
        W = gen_matrix(shape, 4.0, 21)
        M = ops.Q8Matrix.encode(W, local=True, device=dev)
        s = rng.uniform(1e-3, 1e-2, shape[0]).astype(np.float32)
        st = torch.from_numpy(s).to(dev)
        X = torch.from_numpy(rng.standard_normal((64, shape[1])).astype(np.float32)).to(torch.bfloat16).to(dev)
        dY = torch.from_numpy(rng.standard_normal((64, shape[0])).astype(np.float32)).to(torch.bfloat16).to(dev)
        Y = M.matvec_bf16(X, st).double()
        Wd = torch.from_numpy(W).to(dev).double()
        ref = (X.double() @ Wd.T) * st.double()[None, :]
        if not torch.allclose(Y, ref, rtol=1e-4, atol=1e-4 * ref.abs().max().item()):
            raise SystemExit("bench: float forward disagrees with the FP64 product")
        for _ in range(2):
            M.matvec_bf16(X, st)
            M.matvec_t_bf16(dY, st)
    else:
        shape = (16384, 8192) if args.profile_kernel == "dense" else (4096, 4096)
        W = gen_matrix(shape, 4.0, 22)
        x = rng.integers(-127, 128, size=(1, shape[1])).astype(np.int8)
        xd = torch.from_numpy(x).to(dev)
        yref = oracle.matvec_i8(W, x)
        if args.profile_kernel == "awr":
            A = ops.AwrMatrix.encode(W, device=dev)
            run = lambda: A.matvec(xd)
        elif args.profile_kernel == "wpr":
            P = ops.WprMatrix.encode(W, device=dev)
            run = lambda: P.matvec(xd)
        else:
            Wd = torch.from_numpy(W).to(dev)
            x16 = torch.from_numpy(rng.integers(-127, 128, size=(16, shape[1])).astype(np.int8)).to(dev)
            if not np.array_equal(ops.dense_matvec(Wd, x16).cpu().numpy(), oracle.matvec_i8(W, x16.cpu().numpy())):
                raise SystemExit("bench: dense B=16 is not bit-exact")
            run = lambda: (ops.dense_matvec(Wd, xd), ops.dense_matvec(Wd, x16))[0]
        if not np.array_equal(run().cpu().numpy().reshape(1, -1), yref.reshape(1, -1)):
            raise SystemExit(f"bench: {args.profile_kernel} is not bit-exact")
        for _ in range(2):
            run()
    torch.cuda.synchronize()
    ops.device_status()
    return 0


def run_profile_more(args, torch, ops, oracle, dev, rng):
    """More small cases for ncu, each gated first:
    float1    4096x11008 sigma 4, per-row tables, one bf16 vector: forward and re-decoding backward (CUDA cores)
    chain     the 4096 -> 11008 -> 4096 chain (q, gate-shaped, down-shaped matrices) fused in one cooperative launch
    stripes   the reference's ans-warp-stripes layout, 4096x4096 sigma 4, one vector
    fallback  the non-persistent Q8 kernel (columns not a multiple of 16: 4096x4100), one vector"""
    kind = args.profile_kernel
    if kind == "float1":
        shape = (4096, 11008)
        W = gen_matrix(shape, 4.0, 23)
        M = ops.Q8Matrix.encode(W, local=True, device=dev)
        s = torch.from_numpy(rng.uniform(1e-3, 1e-2, shape[0]).astype(np.float32)).to(dev)
        X = torch.from_numpy(rng.standard_normal((1, shape[1])).astype(np.float32)).to(torch.bfloat16).to(dev)
        dY = torch.from_numpy(rng.standard_normal((1, shape[0])).astype(np.float32)).to(torch.bfloat16).to(dev)
        Wd = torch.from_numpy(W).to(dev).double()
        ref = (X.double() @ Wd.T) * s.double()[None, :]
        if not torch.allclose(M.matvec_bf16(X, s).double(), ref, rtol=1e-4, atol=1e-4 * ref.abs().max().item()):
            raise SystemExit("bench: float forward (B=1) disagrees with the FP64 product")
        refb = (dY.double() * s.double()[None, :]) @ Wd
        if not torch.allclose(M.matvec_t_bf16(dY, s).double(), refb, rtol=1e-4, atol=1e-4 * refb.abs().max().item()):
            raise SystemExit("bench: float backward (B=1) disagrees with the FP64 product")
        run = lambda: (M.matvec_bf16(X, s), M.matvec_t_bf16(dY, s))  # noqa: E731
    elif kind == "chain":
        shapes = [(4096, 4096), (11008, 4096), (4096, 11008)]
        Ws = [gen_matrix(sh, 4.0, 30 + i) for i, sh in enumerate(shapes)]
        Ms = [ops.Q8Matrix.encode(W, local=True, device=dev) for W in Ws]
        x0 = torch.from_numpy(rng.integers(-127, 128, size=(1, 4096)).astype(np.int8)).to(dev)
        C = ops.Q8Chain(Ms, [2e-3] * 3, batch=1, x0=x0, device=dev)
        C.run()
        torch.cuda.synchronize()
        v = x0.cpu().numpy()
        for W in Ws:
            y = oracle.matvec_i8(W, v)
            v = np.clip(np.rint(y.astype(np.float32) * np.float32(2e-3)), -128, 127).astype(np.int8)
        if not np.array_equal(C.out8.cpu().numpy(), v):
            raise SystemExit("bench: chain is not bit-exact")
        run = C.run
    elif kind == "stripes":
        W = gen_matrix((4096, 4096), 4.0, 24)
        A = ops.AwsMatrix.encode(W, device=dev)
        x = rng.integers(-127, 128, size=(1, 4096)).astype(np.int8)
        xd = torch.from_numpy(x).to(dev)
        if not np.array_equal(A.matvec(xd).cpu().numpy(), oracle.matvec_i8(W, x)):
            raise SystemExit("bench: stripes kernel is not bit-exact")
        run = lambda: A.matvec(xd)  # noqa: E731
    else:
        W = gen_matrix((4096, 4100), 4.0, 25)
        M = ops.Q8Matrix.encode(W, local=True, device=dev)
        x = rng.integers(-127, 128, size=(1, 4100)).astype(np.int8)
        xd = torch.from_numpy(x).to(dev)
        if not np.array_equal(M.matvec(xd).cpu().numpy(), oracle.matvec_i8(W, x)):
            raise SystemExit("bench: fallback kernel is not bit-exact")
        run = lambda: M.matvec(xd)  # noqa: E731
    for _ in range(2):
        run()
    torch.cuda.synchronize()
    ops.device_status()
    return 0


def run_profile_stack(args):
    """Small fixed stack case for ncu: gate + two plain steps."""
    import torch
    from matvans_b200 import ops
    vals = [int(v) for v in args.profile_stack.split(",")]
    layers, B, engine = vals[:3]
    warps = vals[3] if len(vals) > 3 else 4
    dev = torch.device("cuda", 0)
    mats = build_stack(torch, ops, dev, layers)
    Ms = [m["M"] for m in mats]
    g = torch.Generator(device=dev)
    g.manual_seed(99)
    xs = [torch.randint(-127, 128, (B, M.cols), dtype=torch.int8, device=dev, generator=g) for M in Ms]
    S = ops.Q8Stack(Ms, batch=B, tuning=(warps, 1, 1, 0, 0, engine), xs=xs, device=dev)
    S.run()
    for m, x, y in zip(mats, xs, S.ys):
        if not torch.equal(y, ops.dense_matvec(m["Wd"], x)):
            raise SystemExit(f"bench: {m['spec']['name']} is not bit-exact")
    for _ in range(2):
        S.run()
    torch.cuda.synchronize()
    ops.device_status()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)  # 10 windows of 100 step replays (0.2 s)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-stack", action="store_true",
                    help="skip the 224-matrix batched stack and the large low-entropy sections")
    ap.add_argument("--profile-kernel", default="",
                    choices=["", "awr", "wpr", "dense", "float", "float1", "chain", "stripes", "fallback"],
                    help="small fixed case of one kernel family (the case ncu captures)")
    ap.add_argument("--profile-stack", default="",
                    help="LAYERS,B,ENGINE[,WARPS]: build a stack of LAYERS x 7 matrices and run two steps at B "
                         "vectors with the given engine and warps per CTA (the case ncu captures)")
    ap.add_argument("--tuning", default="", help="fixed stack launch parameters warps,ilp,depth,ctas_per_sm "
                                                  "(default: autotuned)")
    ap.add_argument("--profile", action="store_true",
                    help="run the correctness gate and two steps only (the case ncu captures)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_stack:
        return run_profile_stack(args)
    if args.profile_kernel:
        return run_profile_kernel(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
