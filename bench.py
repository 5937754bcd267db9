"""LigeSIS commit + eval at mu = 24 on B200 (the reference's README row
`LigeSIS 2^7 x 2^17 (mu=24)`, pcs/benches/ligesis.rs:20-60 timing commit and prove).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one `Ligesis::commit` + `Ligesis::prove` of a 2^24-evaluation polynomial arranged as
2^7 x 2^17 (C = 32, eta = 64, s = 128 opened columns, RS rate 1/2, Basefold batched open with
100 queries).  Inputs are seeded synthetic data (uniform Goldilocks f and A, uniform F_{p^2}
point and oracle), the same for every step; f is 128 MiB and the codeword 256 MiB, both larger
than the 126 MB L2, so no step starts from a warm L2.

`value`   device time per step with f already in HBM (lgs_commit_device + lgs_prove; the prove
          includes its small parameter upload and the proof read-back), in ms per proof for the
          whole job (max over ranks / N; N > 1 runs N independent replicas).
`e2e`     the same through the public API (`Ligesis.commit` on a pinned host f, then
          `Ligesis.prove`), host->device copy of f and the proof read-back inside the region.
`--impl reference`: the CPU restatement of the reference prover (oracle/), timed on the same
          mu = 24 workload and inputs, commit and prove separately as
          pcs/benches/ligesis.rs:31-38 times them; its independent loops (rows, columns,
          sumcheck pairs) split over every host core this process may use.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# The line's shape: mu = 24 as 2^7 x 2^17 by default; `--log-m/--log-n` select another
# reference-valid shape (mu = 26 is 2^7 x 2^19).
LOG_M, LOG_N = 7, 17
MU = LOG_M + LOG_N
L2_BYTES = 126 << 20


def metric_for(log_m: int, log_n: int) -> str:
    return f"LigeSIS commit+eval ms at mu={log_m + log_n} (2^{log_m} x 2^{log_n})"


METRIC = metric_for(LOG_M, LOG_N)


def _config(n_gpus: int) -> dict:
    f_mib, cw_mib = (8 << MU) >> 20, (16 << MU) >> 20
    l2 = (f"inputs larger than L2 (f {f_mib} MiB, codeword {cw_mib} MiB); no flush needed"
          if (8 << MU) > L2_BYTES else
          f"inputs smaller than L2 (f {(8 << MU) >> 10} KiB): a test shape, not a bench line")
    return {
        "workload": f"LigeSIS commit+eval, mu={MU} as 2^{LOG_M} x 2^{LOG_N}, C=32, eta=64, s=128, "
                    "RS rate 1/2, Basefold batched open (100 queries)",
        "log_m": LOG_M, "log_n": LOG_N,
        "l2": l2,
        "parallelism": "replicas" if n_gpus > 1 else "single",
    }


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def _max_over_ranks(ms: float, dist, device) -> float:
    """The slowest rank's time (replicas run in parallel, so the job takes the longest one);
    `dist` is torch.distributed after init_process_group, or None for one process."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------------------------------------
# CPU baseline: the oracle (the C++ restatement of the reference prover)
# ------------------------------------------------------------------------------------------------
def bench_inputs(rank: int = 0):
    """The workload's inputs: f (seed 1 + rank), A (seed 2), z (seed 3), oracle arrays (seed 4)."""
    from ligesis_b200 import rng

    f = rng.field_elements(1 + rank, 1 << MU)
    A = rng.field_elements(2, 32 * (64 << LOG_M)).reshape(32, 64 << LOG_M)
    z = rng.ext_elements(3, MU)
    g = rng.SeededRng(4)
    return f, A, z, g.ext_elements(4096), g.ints(4096)


class CpuProver:
    """The oracle's setup, commit and prove on the bench workload.  Setup (the key and its
    Basefold commitment of A) is made once, outside any timing, as pcs/benches/ligesis.rs:28
    times it apart from commit and eval."""

    def __init__(self, threads: int | None = None, rank: int = 0):
        from oracle import orc

        self.orc = orc
        self.threads = orc.set_threads(threads)
        self.f, A, self.z, self.fields, self.ints = bench_inputs(rank)
        self.key = orc.Key(LOG_M, LOG_N, A)

    def step(self) -> tuple[float, float, bytes, bytes]:
        """One commit + prove: (commit s, prove s, root, proof bytes)."""
        t0 = time.perf_counter()
        cm = self.orc.Commitment(self.key, self.f)
        t1 = time.perf_counter()
        proof, _ = self.orc.prove(self.key, cm, self.z, self.fields, self.ints)
        t2 = time.perf_counter()
        return t1 - t0, t2 - t1, cm.root, proof

    def sample_text(self, commit_s: float, prove_s: float, steps: int) -> str:
        return (f"oracle commit+prove on the full mu={MU} workload (2^{LOG_M} x 2^{LOG_N}, same "
                f"inputs as the GPU arm), "
                f"{steps} step(s), mean commit {commit_s:.2f} s + prove {prove_s:.2f} s; "
                f"{self.threads} threads on {_cpu_model()}")


def _cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args) -> None:
    rank, world, _ = _dist()
    if rank != 0:
        return
    cpu = CpuProver()
    for _ in range(args.warmup):
        cpu.step()
    commit_s, prove_s = [], []
    for _ in range(args.steps):
        c, p, _, _ = cpu.step()
        commit_s.append(c)
        prove_s.append(p)
    c_ms, p_ms = statistics.mean(commit_s) * 1e3, statistics.mean(prove_s) * 1e3
    ms = c_ms + p_ms
    line = {
        "metric": metric_for(LOG_M, LOG_N), "value": round(ms, 1), "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 1),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (mod p)",
        "data": "synthetic (seeded uniform Goldilocks)", "config": _config(world),
        "impl": "reference",
        "stages_ms": {"commit": round(c_ms, 1), "prove": round(p_ms, 1)},
        "cpu_baseline": {"value": round(ms, 1), "unit": "ms", "cores": cpu.threads, "kind": "port",
                         "sample": cpu.sample_text(c_ms / 1e3, p_ms / 1e3, args.steps)},
        "e2e": {"value": round(ms, 1), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons of one GPU, read through NVML every ~2 ms on a thread
    while the timed region runs (read-only queries; nothing about the GPU is changed)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, device: int, period_s: float = 0.002):
        self.device, self.period = device, period_s
        self.sm: list[float] = []
        self.mask = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self._nv = None

    def __enter__(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            self._nv = nv
            self._h = nv.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self._h, nv.NVML_CLOCK_SM))
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:
            self._nv = None
        return self

    def _run(self):
        nv = self._nv
        reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)))
                self.mask |= int(reasons(self._h))
            except Exception:
                return
            time.sleep(self.period)

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=2)
        if self._nv:
            try:
                self._nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self) -> dict:
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None,
                "sm_max_mhz": self.max_mhz,
                "reasons": sorted(k for k, bit in self.REASONS.items() if self.mask & bit),
                "samples": len(self.sm)}


# ------------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------------
# DRAM bytes (read + write) per launch of the two commit stages at mu = 24, from one ncu capture
# each (`bench.py --mode commit --steps 3` under ncu --set full; profiles/rs_encode_mu24.md and
# profiles/hash_tc_mu24.md): rs_encode = rs_pass_a + rs_pass_b.
NCU_TRAFFIC_MU24 = {"rs_encode": 842.0e6, "subset_sum_hash": 326.3e6}


def ncu_traffic(stage: str) -> float:
    """Per-launch DRAM bytes of a stage at the line's mu: the mu = 24 capture scaled by 2^(mu-24)
    (both stages stream arrays proportional to 2^mu)."""
    return NCU_TRAFFIC_MU24[stage] * 2.0 ** (MU - 24)


def prove_work(log_m: int, log_n: int) -> dict:
    """Algorithmic HBM bytes and F_{p^2} multiplications of one prove (pcs/src/ligesis.rs:347-549)
    at this shape, item by item: each array is counted once per pass that must touch it.  A
    sumcheck over 2^k entries of S stored factors reads its vectors once per round and writes the
    folded halves: 48 S 2^k bytes; per pair and round it multiplies d + S times (products at the
    evaluation points and the folds).  Kernel-launch latency, partial sums and the proof gather
    are not counted."""
    m, n = 1 << log_m, 1 << log_n
    two_n, W, S = 2 * n, 64 * m, 128
    WS = W * S
    R = max(11 + log_m, log_m + 13, log_n) - 6  # Basefold fold rounds (shared domain)
    D = 2 << R  # Basefold codeword length (rate 1/2)

    def sc(k_len, s_fac, d):
        return 48.0 * s_fac * k_len, (d + s_fac) * k_len  # bytes, EF muls (pairs x 2 rounds)

    items = {
        "abar_gemv": (8.0 * m * n + 16.0 * n, 1.0 * m * n / 2),  # BF x EF = half an EF mul
        "bi_gather_lift": (32.0 * m * S + 8.0 * WS + 2 * (8.0 + 16.0) * WS, 0.0),
        "eq_tables": (16.0 * (WS + WS + n + W), 2.0 * WS + n),
        "sc_binary": sc(WS, 2, 3),
        "sc_bi_batch": sc(WS, 2, 2),
        "sc_hash_recon": tuple(2 * v for v in sc(W, 2, 2)),
        "sc_table": sc(two_n, 2, 2),
        "sc_rslink_a_batch": tuple(2 * v for v in sc(n, 2, 2)),
        "g1_g2_v": (8.0 * 32 * W + 8.0 * WS + 3 * 16.0 * W, 32.0 * W),
        "rs_abar": (16.0 * n + 32.0 * two_n + 2 * 32.0 * two_n, 0.0),
        "basefold_commit_bi": (8.0 * WS * 2 + 16.0 * WS * 3 + 32.0 * D, 0.0),
        "basefold_commit_abar": (16.0 * n * 2 + 32.0 * n * 3 + 32.0 * D, 0.0),
        "batch_open": (8.0 * (32 * W + WS) + 16.0 * n + 16.0 * D * 4, 4.0 * D),
    }
    return {"bytes": sum(v[0] for v in items.values()),
            "ef_muls": sum(v[1] for v in items.values()),
            "items_mb": {k: round(v[0] / 1e6, 2) for k, v in items.items()}}


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "src": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "src": "fallback"}


def run_ours(args) -> None:
    import numpy as np
    import torch

    import ligesis_b200 as L
    from ligesis_b200 import rng

    rank, world, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from ligesis_b200 import autotune

    lib = L.load()
    ctx = L.Context(local)
    tuned = autotune.apply(ctx, LOG_M, LOG_N)  # launch choices from the committed tuning cache
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=torch.device("cuda", local))

    f, A, z, fields, ints = bench_inputs(rank)
    pk, vk = L.Ligesis.setup_with_hash(LOG_M, LOG_N, L.SubsetSumHash(64 << LOG_M, a=A), ctx)
    f_dev = torch.from_numpy(f.view(np.int64)).to(f"cuda:{local}")
    f_pin = torch.from_numpy(f.view(np.int64)).pin_memory()
    f_pin_np = f_pin.numpy().view(np.uint64)
    oracle = L.RandomOracle(0, length=8)
    oracle.fields, oracle.ints = fields, ints

    host_ms = {"commit": 0.0, "prove": 0.0, "n": 0}

    def step_device():
        oracle.restart()
        t0 = time.perf_counter()
        # f is already in HBM and stays there: the commitment reads it in place (no copy)
        commit, data = L.Ligesis.commit_device(pk, f_dev.data_ptr(), f.size, lend=True)
        t1 = time.perf_counter()
        proof = L.Ligesis.prove(pk, data, z, oracle)
        t2 = time.perf_counter()
        host_ms["commit"] += (t1 - t0) * 1e3
        host_ms["prove"] += (t2 - t1) * 1e3
        host_ms["n"] += 1
        return commit, proof

    def step_e2e():
        oracle.restart()
        commit, data = L.Ligesis.commit(pk, L.MlPoly(f_pin_np))
        proof = L.Ligesis.prove(pk, data, z, oracle)
        return commit, proof

    # warm-up; the first proof is checked by the library verifier.  Like the timed loop, it keeps
    # only the previous step's commitment alive while the next one is made, and drops it before
    # the timed region, so the timed steps reuse the buffers the warm-up created.
    prev = None
    for i in range(args.warmup):
        prev = step_device()
        if i == 0:
            oracle.restart()
            assert L.Ligesis.verify(vk, prev[0], z, prev[1], oracle), "warm-up proof rejected"
    del prev

    def timed(fn, k):
        # no cyclic-GC pass of the interpreter inside the timed region (a full collection over
        # torch's object graph takes up to hundreds of ms and lands on whichever step triggers it)
        gc.collect()
        gc.freeze()
        gc.disable()
        if dist:
            dist.barrier()
        torch.cuda.synchronize(local)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        out = None
        for _ in range(k):
            out = fn()
        ev1.record(stream)
        torch.cuda.synchronize(local)
        gc.enable()
        ms = _max_over_ranks(ev0.elapsed_time(ev1) / k, dist, f"cuda:{local}")
        return ms, out

    launches0 = lib.lgs_launch_count()
    host_ms.update(commit=0.0, prove=0.0, n=0)
    L._lib.check(lib.lgs_profile(ctx.handle, 1))
    with ClockSampler(local) as clk:
        dev_ms, (commit, proof) = timed(step_device, args.steps)
    launches = lib.lgs_launch_count() - launches0
    stages = {}
    import ctypes as C

    host_phases = {}
    for name in ("commit_upload", "rs_encode", "subset_sum_hash", "merkle_h", "prove_device",
                 "host_plan", "host_enqueue", "host_wait", "host_assemble"):
        tot, cnt = C.c_double(), C.c_uint64()
        L._lib.check(lib.lgs_profile_get(ctx.handle, name.encode(), C.byref(tot), C.byref(cnt)))
        if cnt.value:
            (host_phases if name.startswith("host_") else stages)[name] = tot.value / cnt.value
    L._lib.check(lib.lgs_profile(ctx.handle, 0))
    root_dev, proof_dev = commit.root, proof.data
    del commit, proof  # the e2e loop reuses these buffers, like the device loop reused the warm-up's
    for _ in range(min(args.warmup, 2)):  # the host-input commit path's first buffers and copies
        step_e2e()
    e2e_ms, (commit2, proof2) = timed(step_e2e, args.steps)
    assert commit2.root == root_dev and proof2.data == proof_dev, "e2e result differs"
    proof = proof2

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    peaks = _peaks()
    # the int8 tensor-core rate of this GPU, measured by the library's own tcgen05 kind::i8
    # microbenchmark (the hash's MMA shape, every SM, back to back)
    i8 = C.c_double()
    L._lib.check(lib.lgs_tensor_peak_i8(ctx.handle, 32768, C.byref(i8)))
    # roofline of the dominant kernel stage
    n, two_n, W = 1 << LOG_N, 2 << LOG_N, 64 << LOG_M
    m = 1 << LOG_M
    hash_ops = 2.0 * 256 * W * two_n  # int8 MACs x 2 over 8 limbs x 32 rows
    ntt_bytes = 8.0 * m * n + 8.0 * m * two_n
    dom = max(("subset_sum_hash", "rs_encode"), key=lambda s: stages.get(s, 0.0))
    if dom == "subset_sum_hash":
        ach = hash_ops / (stages[dom] * 1e-3) / 1e12
        peak = i8.value
        roof = {"kernel": "subset_sum_hash (hash_tc_kernel)", "bound": "tensor",
                "achieved": round(ach, 1), "peak": round(peak, 1), "unit": "TOP/s (int8)",
                "frac": round(ach / peak, 4), "traffic": ncu_traffic("subset_sum_hash"),
                "peak_src": "measured: tcgen05.mma kind::i8 M128N256K32 from shared memory on "
                            "every SM (lgs_tensor_peak_i8)",
                "algorithmic": f"{hash_ops:.3e} int8 ops per launch"}
    else:
        ach = ntt_bytes / (stages[dom] * 1e-3) / 1e9
        peak = peaks["hbm_gbs"]
        roof = {"kernel": "rs_encode (rs_pass_a + rs_pass_b)", "bound": "hbm",
                "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": ncu_traffic("rs_encode"),
                "peak_src": ("measured HBM copy (MEASURED_PEAKS.json)" if peaks["src"] == "measured"
                             else "fallback: 6.65 TB/s, an earlier copy measurement on this pool "
                                  "(MEASURED_PEAKS.json absent)"),
                "algorithmic": f"{ntt_bytes:.3e} bytes per launch"}
    others = {}
    if "rs_encode" in stages:
        a = ntt_bytes / (stages["rs_encode"] * 1e-3) / 1e9
        others["rs_encode"] = {"bound": "hbm", "achieved": round(a, 1), "unit": "GB/s",
                               "peak": peaks["hbm_gbs"], "frac": round(a / peaks["hbm_gbs"], 4),
                               "traffic": ncu_traffic("rs_encode"),
                               "alu_floor": rs_alu_floor(lib, ctx, LOG_M, LOG_N,
                                                         stages["rs_encode"])}
    if "subset_sum_hash" in stages:
        a = hash_ops / (stages["subset_sum_hash"] * 1e-3) / 1e12
        others["subset_sum_hash"] = {"bound": "tensor", "achieved": round(a, 1),
                                     "unit": "TOP/s (int8)", "peak": round(i8.value, 1),
                                     "frac": round(a / i8.value, 4),
                                     "traffic": ncu_traffic("subset_sum_hash")}

    if "prove_device" in stages:
        pw = prove_work(LOG_M, LOG_N)
        t = stages["prove_device"] * 1e-3
        a = pw["bytes"] / t / 1e9
        others["prove_device"] = {
            "bound": "hbm", "achieved": round(a, 1), "unit": "GB/s", "peak": peaks["hbm_gbs"],
            "frac": round(a / peaks["hbm_gbs"], 4), "traffic": None,
            "algorithmic": f"{pw['bytes']:.3e} bytes, {pw['ef_muls']:.3e} F_p2 muls per prove",
            "ef_muls_per_s": round(pw["ef_muls"] / t / 1e9, 2), "items_mb": pw["items_mb"],
            "note": "the prove's time inside the step (beside the commit's hash and tree)"}

    cpu = None
    if not args.no_cpu_baseline and world == 1:
        # one full step of the same workload (not scaled); its root and proof must equal ours
        cp = CpuProver(rank=rank)
        c_s, p_s, c_root, c_proof = cp.step()
        assert c_root == root_dev and c_proof == proof_dev, "oracle and GPU proofs differ"
        cpu = {"value": round((c_s + p_s) * 1e3, 1), "unit": "ms", "cores": cp.threads,
               "kind": "port", "sample": cp.sample_text(c_s, p_s, 1)}

    extra = {}
    if world == 1 and not args.no_batch_serve:
        # the batched and served forms of the same prover, beside the one-at-a-time path
        extra["batch"] = batch_stats(args.lanes)
        extra["serve"] = serve_stats(args.requests, args.rate, args.lanes)

    value = dev_ms / world
    line = {
        "metric": metric_for(LOG_M, LOG_N), "value": round(value, 3), "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dev_ms, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (mod p)",
        "data": "synthetic (seeded uniform Goldilocks)",
        "config": {**_config(world), "tuning": tuned or "built-in defaults"},
        "e2e": {"value": round(e2e_ms / world, 3), "unit": "ms",
                "h2d_bytes_per_step": int(f.nbytes), "d2h_bytes_per_step": len(proof.data) + 32},
        "stages_ms": {k: round(v, 4) for k, v in stages.items()},
        "host_wall_ms": {k: round(host_ms[k] / max(host_ms["n"], 1), 4) for k in ("commit", "prove")},
        "prove_host_phases_ms": {k[5:]: round(v, 4) for k, v in host_phases.items()},
        "roofline": roof,
        "stage_rooflines": others,
        "cpu_baseline": cpu,
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "proof_bytes": len(proof.data), "proof_size_bytes_ref_accounting": proof.size_bytes(),
        **extra,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------
# batched and served proving (not part of the default line)
# ------------------------------------------------------------------------------------------------
def _keys_for(mus, ctx):
    import ligesis_b200 as L
    from ligesis_b200 import rng
    from ligesis_b200.workloads import shape_for_mu

    keys = {}
    for mu in sorted(set(mus)):
        lm, ln = shape_for_mu(mu)
        A = rng.field_elements(100 + lm, 32 * (64 << lm)).reshape(32, 64 << lm)  # one A per m
        keys[mu] = L.Ligesis.setup_with_hash(lm, ln, L.SubsetSumHash(64 << lm, a=A), ctx)[0]
    return keys


def rs_alu_floor(lib, ctx, log_m: int, log_n: int, measured_ms: float) -> dict:
    """The RS encoding's arithmetic floor: its radix-8 DFTs and twiddle multiplications (counted
    from the kernels' structure, rs_dft.cu) at the device-wide rates of lgs_rs_alu_rates, which
    run the same arithmetic with no memory traffic."""
    import ctypes as C
    import math

    r8, mul = C.c_double(), C.c_double()
    import ligesis_b200 as L

    L._lib.check(lib.lgs_rs_alu_rates(ctx.handle, 4096, C.byref(r8), C.byref(mul)))
    N = 2 << log_n
    n2 = N >> 12
    # pass A: four radix-8 stages (the first on a half-zero input, 8 of its 12 butterflies),
    # 7 + 8 + 7 twiddle products per 8 values; pass B: log8(N2) stages, 15 products per 8
    # values when N2 = 64 (one per value otherwise)
    r8_per = (2.0 / 3.0 + 3.0) / 8.0 + (math.log2(n2) / 3.0) / 8.0
    mul_per = 22.0 / 8.0 + (15.0 / 8.0 if n2 == 64 else 1.0)
    values = float(1 << log_m) * N
    floor_ms = values * (r8_per / r8.value + mul_per / mul.value) * 1e3
    return {"floor_ms": round(floor_ms, 4), "frac_of_floor": round(floor_ms / measured_ms, 4),
            "radix8_per_s": round(r8.value, 1), "mul_per_s": round(mul.value, 1),
            "radix8_per_value": round(r8_per, 4), "mul_per_value": round(mul_per, 4),
            "note": "arithmetic only (registers, no loads, stores or exchanges): the time the "
                    "encoding's butterflies and twiddle products take at full occupancy"}


def batch_stats(lanes: int, reps: int = 7) -> dict:
    """96 polynomials of uneven size (mu = floor(14 + 8u)), each committed and opened at its own
    point: one at a time on one context versus all through the engine's lanes; host f in, proof
    out.  Each side is timed `reps` times and the best run counts; every proof of the engine must
    equal the one-at-a-time proof."""
    import ligesis_b200 as L
    from ligesis_b200 import rng
    from ligesis_b200.engine import ProverEngine
    from ligesis_b200.workloads import batch_mus

    mus = batch_mus(96)
    ctx = L.Context(0)
    keys = _keys_for(mus, ctx)
    jobs = []
    for i, mu in enumerate(mus):
        f = rng.field_elements(1000 + i, 1 << mu)
        z = rng.ext_elements(2000 + i, mu)
        jobs.append((keys[mu], f, z, 3000 + i))

    # the pre-drawn oracles are inputs like f and z: built before any timed region
    oracles = [L.RandomOracle(os_, length=1024) for _, _, _, os_ in jobs]

    def plain():
        out = []
        for (pk, f, z, _), o in zip(jobs, oracles):
            o.restart()
            c, d = L.Ligesis.commit(pk, L.MlPoly(f))
            out.append((c.root, L.Ligesis.prove(pk, d, z, o).data))
        return out

    def batched(eng):
        for o in oracles:
            o.restart()
        res = eng.run([(pk, f, z, o) for (pk, f, z, _), o in zip(jobs, oracles)])
        return [(r.commit.root, r.proof.data) for r in res]

    def best(fn):
        t_best, out = None, None
        for _ in range(reps):
            gc.collect()
            gc.freeze()
            gc.disable()
            t0 = time.perf_counter()
            out = fn()
            t = time.perf_counter() - t0
            gc.enable()
            t_best = t if t_best is None else min(t_best, t)
        return t_best, out

    plain()  # warm-up: arenas and pools of every shape
    t_plain, ref = best(plain)
    with ProverEngine(0, lanes=lanes) as eng:
        tuning = eng.tuning
        eng.prepare(keys.values())
        batched(eng)
        t_batch, got = best(lambda: batched(eng))
    return {"jobs": len(jobs), "mu": [min(mus), max(mus)], "lanes": lanes,
            "lane_tuning": tuning or "built-in defaults",
            "plain_proofs_per_s": round(len(jobs) / t_plain, 1),
            "batched_proofs_per_s": round(len(jobs) / t_batch, 1),
            "speedup": round(t_plain / t_batch, 2), "identical_proofs": got == ref,
            "timing": f"host wall clock, best of {reps}, host f in, proof out (end to end)"}


def run_batch(args) -> None:
    print(json.dumps({"mode": "batch", **batch_stats(args.lanes)}), flush=True)


def serve_stats(requests: int, rate: float, lanes: int) -> dict:
    """A Poisson stream of commit+eval requests (mean `rate`/s, mu in [14, 24], 10% GPT-2 layer
    witnesses): latency percentiles and proofs/s for the one-at-a-time path (1 lane) and the
    engine (many lanes), plus both when every request is queued at once (peak throughput)."""
    import threading as th

    import numpy as np

    import ligesis_b200 as L
    from ligesis_b200 import rng
    from ligesis_b200.engine import ProverEngine
    from ligesis_b200.workloads import gpt2_layer_witness, serve_stream

    stream = serve_stream(requests, rate_per_s=rate)
    mus = [mu for _, mu, _ in stream]
    ctx = L.Context(0)
    keys = _keys_for(mus, ctx)
    f_by_mu = {mu: rng.field_elements(4000 + mu, 1 << mu) for mu in set(mus)}
    gpt2 = gpt2_layer_witness()
    reqs = []
    for i, (t, mu, kind) in enumerate(stream):
        f = gpt2 if kind == "gpt2" else f_by_mu[mu]
        # the pre-drawn oracle is an input of the request, like f and z
        reqs.append((t, keys[mu], f, rng.ext_elements(5000 + i, mu),
                     L.RandomOracle(6000 + i, length=1024)))

    def drive(lanes: int, paced: bool):
        with ProverEngine(0, lanes=lanes) as eng:
            eng.prepare(keys.values())
            for _, pk, f, z, o in reqs[: 2 * lanes]:  # warm every lane
                o.restart()
                eng.wait(eng.submit(pk, f, z, o))
            for r in reqs:
                r[4].restart()
            results = [None] * len(reqs)
            tickets = [None] * len(reqs)
            ready = th.Semaphore(0)

            def collect():
                for i in range(len(reqs)):
                    ready.acquire()
                    results[i] = eng.wait(tickets[i])

            col = th.Thread(target=collect)
            gc.collect()
            gc.freeze()
            gc.disable()
            col.start()
            start = time.perf_counter()
            for i, (t, pk, f, z, o) in enumerate(reqs):
                if paced:
                    delay = start + t - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                tickets[i] = eng.submit(pk, f, z, o)
                ready.release()
            col.join()
            wall = time.perf_counter() - start
            gc.enable()
        lat = np.array([r.latency_ms for r in results])
        return {"proofs_per_s": round(len(reqs) / wall, 1),
                "p50_ms": round(float(np.percentile(lat, 50)), 2),
                "p99_ms": round(float(np.percentile(lat, 99)), 2)}, [r.proof.data for r in results]

    plain_paced, ref = drive(1, True)
    eng_paced, got = drive(lanes, True)
    plain_peak, _ = drive(1, False)
    eng_peak, got2 = drive(lanes, False)
    return {"requests": len(reqs), "arrival_rate_per_s": rate,
            "mu": [min(mus), max(mus)], "gpt2_requests": sum(1 for r in stream if r[2] == "gpt2"),
            "lanes": lanes, "plain": plain_paced, "served": eng_paced,
            "plain_saturated": plain_peak, "served_saturated": eng_peak,
            "throughput_ratio_saturated": round(eng_peak["proofs_per_s"] / plain_peak["proofs_per_s"], 2),
            "identical_proofs": got == ref and got2 == ref,
            "timing": "latency = engine clock from submission (arrival) to proof; host f in"}


def run_serve(args) -> None:
    print(json.dumps({"mode": "serve", **serve_stats(args.requests, args.rate, args.lanes)}),
          flush=True)


def run_commit(args) -> None:
    """Commit only (RS encode, subset-sum hash with its leaf hashes, Merkle tree) of a polynomial
    already in HBM, `--steps` times after warm-up, per shape: the square shapes 2^10 x 2^10,
    2^12 x 2^12 and 2^13 x 2^13 (mu = 20, 24, 26) that setup's shared-domain window rejects run
    through the commit-only key.  Also the case the per-kernel ncu captures of the commit
    kernels run (--shapes 7x17)."""
    import ctypes as C

    import numpy as np
    import torch

    import ligesis_b200 as L
    from ligesis_b200 import rng

    shapes = [tuple(int(v) for v in sh.split("x")) for sh in args.shapes.split(",")]
    lib = L.load()
    ctx = L.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=torch.device("cuda", 0))
    peaks = _peaks()
    i8 = C.c_double()
    L._lib.check(lib.lgs_tensor_peak_i8(ctx.handle, 32768, C.byref(i8)))
    for lm, ln in shapes:
        f = rng.field_elements(1, 1 << (lm + ln))
        A = rng.field_elements(2, 32 * (64 << lm)).reshape(32, 64 << lm)
        hsh = L.SubsetSumHash(64 << lm, a=A)
        full = L.shape_ok(lm, ln)
        pk = (L.Ligesis.setup_with_hash(lm, ln, hsh, ctx)[0] if full
              else L.Ligesis.setup_commit_only(lm, ln, hsh, ctx))
        f_dev = torch.from_numpy(f.view(np.int64)).to("cuda:0")
        roots = set()
        for _ in range(args.warmup):
            commit, data = L.Ligesis.commit_device(pk, f_dev.data_ptr(), f.size)
            roots.add(commit.root)
            del data
        L._lib.check(lib.lgs_profile(ctx.handle, 1))
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            commit, data = L.Ligesis.commit_device(pk, f_dev.data_ptr(), f.size)
            roots.add(commit.root)  # waits for the commit's hash stream too
            del data
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
        stages = {}
        for name in ("rs_encode", "subset_sum_hash", "merkle_h"):
            tot, cnt = C.c_double(), C.c_uint64()
            L._lib.check(lib.lgs_profile_get(ctx.handle, name.encode(), C.byref(tot), C.byref(cnt)))
            if cnt.value:
                stages[name] = round(tot.value / cnt.value, 4)
        L._lib.check(lib.lgs_profile(ctx.handle, 0))
        m, n = 1 << lm, 1 << ln
        W, two_n = 64 * m, 2 * n
        ntt_gbs = (8.0 * m * n + 8.0 * m * two_n) / (stages["rs_encode"] * 1e-3) / 1e9
        hash_tops = 2.0 * 256 * W * two_n / (stages["subset_sum_hash"] * 1e-3) / 1e12
        merkle_gbs = (256.0 * two_n + 64.0 * (two_n - 1)) / (stages["merkle_h"] * 1e-3) / 1e9
        print(json.dumps({
            "mode": "commit", "metric": f"LigeSIS commit ms at mu={lm + ln} (2^{lm} x 2^{ln})",
            "value": round(ms, 4), "unit": "ms", "log_m": lm, "log_n": ln,
            "key": "setup" if full else "commit-only (outside setup's shared-domain window)",
            "steps": args.steps, "warmup": args.warmup, "stages_ms": stages,
            "ntt_gbs": round(ntt_gbs, 1), "ntt_frac_hbm": round(ntt_gbs / peaks["hbm_gbs"], 4),
            "hash_int8_tops": round(hash_tops, 1),
            "hash_frac_int8": round(hash_tops / i8.value, 4),
            "merkle_input_gbs": round(merkle_gbs, 1), "roots_identical": len(roots) == 1,
            "timing": "CUDA events on the library stream; f resident in HBM"}), flush=True)
        del pk, f_dev, commit


def run_sumcheck(args) -> None:
    """The reference's sumcheck microbenchmark (pcs/benches/sumcheck.rs:64-68: a product of 3
    multilinears) over F_{p^2} at mu = 20, 22, 24, device-resident factors; the eq-product
    variant [eq_z, f, g] (eq_z built on the device first, inside the timing); and an MlPoly
    new_eq / fold (one variable) / eval sweep.  Each timed call gets fresh inputs: the factors
    are folded in place, so they are restored from a pristine copy between calls, outside the
    CUDA events.  Bytes are algorithmic: the sumcheck reads its 3 x 16 B factors once per round
    and writes the folded half (48 d B per element over all rounds, d factors); new_eq writes 16 B per
    entry, fold reads 16 B and writes 8 B per input entry, eval reads 16 B per entry."""
    import numpy as np
    import torch

    import ligesis_b200 as L
    from ligesis_b200 import rng

    lib = L.load()
    ctx = L.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=torch.device("cuda", 0))
    peaks = _peaks()
    mus = [int(v) for v in args.mus.split(",")]
    d = args.sc_d

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int64).reshape(-1)).to("cuda:0")

    def timed(fn, prep=None):
        tot = 0.0
        for i in range(args.warmup + args.steps):
            if prep:
                prep()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            if i >= args.warmup:
                tot += e0.elapsed_time(e1)
        return tot / args.steps

    def line(op, mu, ms, nbytes, **kw):
        gbs = nbytes / (ms * 1e-3) / 1e9
        print(json.dumps({"mode": "sumcheck", "op": op, "mu": mu, "value": round(ms, 4),
                          "unit": "ms", "gbs": round(gbs, 1),
                          "frac_hbm": round(gbs / peaks["hbm_gbs"], 4), "steps": args.steps,
                          "warmup": args.warmup, **kw}), flush=True)

    for mu in mus:
        n = 1 << mu
        pristine = dev(np.concatenate([rng.ext_elements(9000 + j, n) for j in range(d)]))
        work = torch.empty_like(pristine)
        ch = dev(rng.ext_elements(9100 + mu, mu))
        z = dev(rng.ext_elements(9200 + mu, mu))
        rounds = torch.zeros(mu * (d + 1) * 2, dtype=torch.int64, device="cuda:0")
        finals = torch.zeros(d * 2, dtype=torch.int64, device="cuda:0")

        def restore():
            work.copy_(pristine)

        def sc():
            L._lib.check(lib.lgs_sumcheck_prove_dev(ctx.handle, work.data_ptr(), d, mu,
                                                    ch.data_ptr(), rounds.data_ptr(),
                                                    finals.data_ptr()))

        ms = timed(sc, restore)
        line(f"sumcheck_{d}", mu, ms, 48.0 * d * n,
             ef_muls_per_s=round((d + 1 + 2 * d) * n / (ms * 1e-3) / 1e9, 2))

        def eq_variant():
            L._lib.check(lib.lgs_new_eq_dev(ctx.handle, z.data_ptr(), mu, work.data_ptr()))
            sc()

        if d == 3:
            ms = timed(eq_variant, restore)
            line("sumcheck_eq_f_g", mu, ms, 144.0 * n + 16.0 * n)

        out = torch.empty(2 * n, dtype=torch.int64, device="cuda:0")
        ms = timed(lambda: L._lib.check(lib.lgs_new_eq_dev(ctx.handle, z.data_ptr(), mu,
                                                           out.data_ptr())))
        line("new_eq", mu, ms, 16.0 * n)
        ms = timed(lambda: L._lib.check(lib.lgs_mle_fold_dev(ctx.handle, pristine.data_ptr(), mu,
                                                             z.data_ptr(), 1, out.data_ptr())))
        line("fold_1", mu, ms, 24.0 * n)
        val = torch.zeros(2, dtype=torch.int64, device="cuda:0")
        ms = timed(lambda: L._lib.check(lib.lgs_mle_eval_dev(ctx.handle, pristine.data_ptr(), mu,
                                                             z.data_ptr(), val.data_ptr())))
        line("eval", mu, ms, 16.0 * n)
        del pristine, work, out


def run_autotune(args) -> None:
    """Times candidate launch choices of the commit + prove step and records the fastest in
    ligesis_b200/tuning.json (see ligesis_b200/autotune.py)."""
    from ligesis_b200 import autotune

    entry = autotune.tune(args.log_m, args.log_n, steps=args.steps, warmup=args.warmup)
    print(json.dumps({"mode": "autotune", "log_m": args.log_m, "log_n": args.log_n, **entry}),
          flush=True)
    if args.engine:  # the engine lanes' launch choices on the batch workload
        entry = autotune.tune_engine(lanes=args.lanes)
        print(json.dumps({"mode": "autotune", "engine": args.lanes, **entry}), flush=True)


def run_timeline(args) -> None:
    """The prove's replayed graph with timeline event nodes (profile level 2): for each branch
    boundary, ms from the prove's start, averaged over `--steps` proves of one commitment.  With
    --overlap each prove follows a fresh commit of the same polynomial, as in the bench step, so
    the commit's hash and tree run beside it."""
    import numpy as np
    import torch

    import ligesis_b200 as L
    from ligesis_b200 import rng

    lm, ln = args.log_m, args.log_n
    lib = L.load()
    ctx = L.Context(0)
    f = rng.field_elements(1, 1 << (lm + ln))
    A = rng.field_elements(2, 32 * (64 << lm)).reshape(32, 64 << lm)
    z = rng.ext_elements(3, lm + ln)
    g = rng.SeededRng(4)
    oracle = L.RandomOracle(0, length=8)
    oracle.fields, oracle.ints = g.ext_elements(4096), g.ints(4096)
    pk, _ = L.Ligesis.setup_with_hash(lm, ln, L.SubsetSumHash(64 << lm, a=A), ctx)
    from ligesis_b200 import autotune

    if args.overlap:
        autotune.apply(ctx, lm, ln)
    f_dev = torch.from_numpy(f.view(np.int64)).to("cuda:0")
    commit, data = L.Ligesis.commit_device(pk, f_dev.data_ptr(), f.size)
    import ctypes as C

    def one():
        nonlocal commit, data
        if args.overlap:
            del data
            commit, data = L.Ligesis.commit_device(pk, f_dev.data_ptr(), f.size)
        oracle.restart()
        L.Ligesis.prove(pk, data, z, oracle)

    L._lib.check(lib.lgs_profile(ctx.handle, 2))
    for _ in range(3):  # eager, capture, first replay
        one()
    L._lib.check(lib.lgs_profile(ctx.handle, 2))
    for _ in range(args.steps):
        one()
    need = C.c_size_t()
    L._lib.check(lib.lgs_profile_names(ctx.handle, None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    L._lib.check(lib.lgs_profile_names(ctx.handle, buf, need.value, C.byref(need)))
    names = [nm for nm in buf.value.decode().split("\n") if nm.startswith("tl:")]
    out = {}
    for name in ["prove_device"] + names:
        tot, cnt = C.c_double(), C.c_uint64()
        L._lib.check(lib.lgs_profile_get(ctx.handle, name.encode(), C.byref(tot), C.byref(cnt)))
        if cnt.value:
            out[name] = round(tot.value / cnt.value, 4)
    out = dict(sorted(out.items(), key=lambda kv: kv[1]))
    print(json.dumps({"mode": "timeline", "log_m": lm, "log_n": ln, "proves": args.steps,
                      "ms_from_prove_start": out, "root": commit.root.hex()[:16]}), flush=True)


def run_basefold(args) -> None:
    """Standalone Basefold (pcs/benches/basefold.rs:144-150: mu in {22, 24}, code_rate 1, BF,
    log_interleave 6): device commit (host polynomial in, root out), prove (host point and oracle
    in, proof bytes out) and host verify, each the mean of `--steps` runs after warm-up; the CPU
    oracle's commit and prove at mu = 22 beside it, and the README's single-thread numbers
    (README.md:172,174) for context."""
    import numpy as np

    import ligesis_b200 as L
    from ligesis_b200 import rng

    ctx = L.Context(0)
    readme = {22: {"commit_s": 1.0, "eval_s": 0.85, "verify_s": 0.007, "proof_kb": 391},
              24: {"commit_s": 5.0, "eval_s": 3.5, "verify_s": 0.009, "proof_kb": 527}}
    out = {}
    for mu in (22, 24):
        poly = L.MlPoly(rng.field_elements(10 + mu, 1 << mu))
        pt = rng.ext_elements(20 + mu, mu)
        oracle = L.RandomOracle(30 + mu, length=1024)
        for _ in range(args.warmup):
            state, commit = L.Basefold.commit_base(poly, 1, ctx)
            oracle.restart()
            proof = L.Basefold.prove(state, pt, oracle)
        gc.collect()
        gc.disable()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            del state
            state, commit = L.Basefold.commit_base(poly, 1, ctx)
        t1 = time.perf_counter()
        for _ in range(args.steps):
            oracle.restart()
            proof = L.Basefold.prove(state, pt, oracle)
        t2 = time.perf_counter()
        for _ in range(args.steps):
            oracle.restart()
            ok = L.Basefold.verify(commit, pt, proof, oracle)
        t3 = time.perf_counter()
        gc.enable()
        assert ok, "Basefold proof rejected"
        k = args.steps
        out[mu] = {"commit_ms": round((t1 - t0) / k * 1e3, 3), "prove_ms": round((t2 - t1) / k * 1e3, 3),
                   "verify_ms": round((t3 - t2) / k * 1e3, 3), "proof_bytes": len(proof),
                   "readme_cpu_1thread": readme[mu]}
        del state
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import orc

        poly = rng.field_elements(32, 1 << 22)
        t0 = time.perf_counter()
        cm = orc.BasefoldCommitment(poly, False, 1, 6)
        t1 = time.perf_counter()
        g = rng.SeededRng(52)
        orc.basefold_prove(cm, rng.ext_elements(42, 22), g.ext_elements(1024), g.ints(1024))
        t2 = time.perf_counter()
        cpu = {"mu": 22, "commit_ms": round((t1 - t0) * 1e3, 1), "prove_ms": round((t2 - t1) * 1e3, 1),
               "cores": 1, "kind": "port", "cpu": _cpu_model()}
    print(json.dumps({"mode": "basefold", "code_rate": 1, "log_interleave": 6, "steps": args.steps,
                      "timing": "host wall clock per call: host polynomial / point in, root / "
                                "proof bytes out", "gpu": out, "cpu_oracle": cpu}), flush=True)


def _field_sub(x, a):
    """x - a mod p elementwise (x a canonical scalar, a canonical uint64 array)."""
    import numpy as np

    p = np.uint64(0xFFFFFFFF00000001)
    d = p - a  # in (0, p]
    s = np.uint64(x) + d
    s = np.where(s < d, s + np.uint64(0xFFFFFFFF), s)  # wrapped: add 2^64 mod p
    return np.where(s >= p, s - p, s)


def run_logup(args) -> None:
    """GKR-LogUp lookup (logup/benches/logup.rs:33-79: m = 2^mu queries into an n = 2^nu table,
    multiplicities precomputed, (mu, nu) in {(20, 14), (22, 16)}): lookup prove from host arrays
    (copies in the timed call), from device-resident tensors, and the query-side fraction sum
    alone (the m-sized pass that dominates), each the mean of `--steps` calls after warm-up; host
    verify; the CPU oracle's lookup prove at (20, 14) beside it."""
    import numpy as np
    import torch

    import ligesis_b200 as L
    from ligesis_b200 import rng

    ctx = L.Context(0)
    out = {}
    shapes = ((20, 14), (22, 16)) if args.mu is None else ((args.mu, args.nu),)
    for mu, nu in shapes:
        t = rng.ext_elements(70 + nu, 1 << nu)
        idx = (rng.ints(71 + mu, 1 << mu) % np.uint64(1 << nu)).astype(np.int64)
        a = t[idx]
        e = L.multiplicity_vector(a, t)
        fields = rng.ext_elements(72 + mu, 1024)
        oracle = L.RandomOracle(0, length=4)
        oracle.fields = np.ascontiguousarray(fields)
        dev = [torch.from_numpy(x.view(np.int64)).cuda() for x in (a, t, e)]
        qq = np.stack([_field_sub(fields[0][c], a[:, c]) for c in (0, 1)], 1)
        qq_dev = torch.from_numpy(np.ascontiguousarray(qq).view(np.int64)).cuda()
        torch.cuda.synchronize()

        def host_call():
            oracle.restart()
            return L.Lookup.prove_with_mults(a, t, e, oracle, ctx)

        def dev_call():
            oracle.restart()
            return L.Lookup.prove_with_mults(*dev, oracle, ctx)

        def query_call():
            oracle.restart()
            return L.FracSum.prove(None, qq_dev, oracle, ctx)

        res = {}
        for name, fn in (("prove_host_inputs_ms", host_call), ("prove_device_inputs_ms", dev_call),
                         ("query_frac_sum_device_ms", query_call)):
            for _ in range(args.warmup):
                r = fn()
            gc.collect()
            gc.disable()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                r = fn()
            t1 = time.perf_counter()
            gc.enable()
            res[name] = round((t1 - t0) / args.steps * 1e3, 3)
        proof = host_call()
        oracle.restart()
        t0 = time.perf_counter()
        claims = L.Lookup.verify(proof, oracle)
        res["verify_ms"] = round((time.perf_counter() - t0) * 1e3, 3)
        assert claims is not None, "lookup proof rejected"
        res["proof_bytes"] = proof.size_bytes()
        res["h2d_bytes"] = int(a.nbytes + t.nbytes + e.nbytes)
        out[f"mu{mu}_nu{nu}"] = res
        del dev, qq_dev
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import orc

        mu, nu = 20, 14
        t = rng.ext_elements(70 + nu, 1 << nu)
        idx = (rng.ints(71 + mu, 1 << mu) % np.uint64(1 << nu)).astype(np.int64)
        a = t[idx]
        e = L.multiplicity_vector(a, t)
        fields = rng.ext_elements(72 + mu, 1024)
        t0 = time.perf_counter()
        orc.lookup_prove(a, t, e, fields)
        cpu = {"mu": mu, "nu": nu, "prove_ms": round((time.perf_counter() - t0) * 1e3, 1),
               "cores": 1, "kind": "port", "cpu": _cpu_model()}
    print(json.dumps({"mode": "logup", "steps": args.steps,
                      "timing": "host wall clock per call, proof bytes out", "gpu": out,
                      "cpu_oracle": cpu}), flush=True)


def run_witness(args) -> None:
    """proofsys' rescaled linear layers of the integer GPT-2 (Config::gpt2_31: 31 positions,
    d_model 768, MLP 3072, vocabulary 50257, scale 2^12; model.rs:360-374, :225-228) on the GPU:
    each layer shape from host arrays (copies in the timed call) and from device tensors, the
    whole forward's linear work (12 blocks x (qkv, attention projection, fc, fproj) + the
    vocabulary head), and the oracle's time for one MLP fc layer.  Seeded synthetic values:
    activations within +-max_v * scale, weights within +-2^15 (no exported model here)."""
    import numpy as np
    import torch

    import ligesis_b200 as L
    from ligesis_b200 import proofsys as ps

    ctx = L.Context(0)
    cfg = ps.GPT2_31
    n, d, h, v, sc = cfg["n_seq"], cfg["d_model"], cfg["mlp_hidden"], cfg["vocab"], cfg["scale"]
    g = np.random.default_rng(8)
    act = cfg["max_v"] * sc
    shapes = {"qkv": (d, 3 * d, False), "attn_proj": (d, d, False), "fc": (d, h, False),
              "fproj": (h, d, False), "vocab_head": (d, v, True)}
    if args.layer:
        shapes = {args.layer: shapes[args.layer]}
    out = {}
    for name, (inner, cols, wt) in shapes.items():
        x = g.integers(-act, act, size=(n, inner), dtype=np.int64)
        w = g.integers(-(1 << 15), 1 << 15, size=(cols, inner) if wt else (inner, cols),
                       dtype=np.int64)
        b = g.integers(-act, act, size=cols, dtype=np.int64)
        xd, wd, bd = (torch.from_numpy(a).cuda() for a in (x, w, b))
        res = {}
        for label, fn in (("host_ms", lambda: ps.linear_witness(x, w, b, sc, wt, ctx)),
                          ("device_ms", lambda: ps.linear_witness(xd, wd, bd, sc, wt, ctx))):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                fn()
            torch.cuda.synchronize()
            res[label] = round((time.perf_counter() - t0) / args.steps * 1e3, 3)
        # the contraction kernel alone (CUDA events around it, device operands)
        import ctypes as C

        lib = L.load()
        L._lib.check(lib.lgs_profile(ctx.handle, 1))
        for _ in range(args.steps):
            ps.linear_witness(xd, wd, bd, sc, wt, ctx)
        for stage in ("linear_witness_tc", "linear_witness_cores"):
            tot, cnt = C.c_double(), C.c_uint64()
            L._lib.check(lib.lgs_profile_get(ctx.handle, stage.encode(), C.byref(tot),
                                             C.byref(cnt)))
            if cnt.value:
                res[stage + "_kernel_ms"] = round(tot.value / cnt.value, 4)
        L._lib.check(lib.lgs_profile(ctx.handle, 0))
        kern = res.get("linear_witness_tc_kernel_ms")
        if kern:
            # HBM bytes: the weights and activations read once, four outputs written
            bytes_ = 8.0 * (inner * cols + n * inner + 4 * n * cols)
            res["kernel_gbs"] = round(bytes_ / (kern * 1e-3) / 1e9, 1)
            res["kernel_frac_hbm"] = round(res["kernel_gbs"] / _peaks()["hbm_gbs"], 4)
        res["products"] = n * inner * cols
        out[name] = res
    if args.layer:
        print(json.dumps({"mode": "witness", "config": "gpt2_31", "steps": args.steps,
                          "timing": "host wall clock per call", "layers": out}), flush=True)
        return
    forward = 12 * sum(out[k]["device_ms"] for k in ("qkv", "attn_proj", "fc", "fproj")) \
        + out["vocab_head"]["device_ms"]
    # one whole block's witness (layer norms, attention with 12 heads, softmax, MLP, GELU
    # lookup), host arrays in and out, every step on the GPU
    bcfg = dict(cfg, n_head=12)
    bx, bw, bel, bgl = ps.synthetic_block(12, bcfg)
    for _ in range(args.warmup):
        ps.block_witness(bx, bw, bel, bgl, bcfg, ctx)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ps.block_witness(bx, bw, bel, bgl, bcfg, ctx)
    block_ms = round((time.perf_counter() - t0) / args.steps * 1e3, 3)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import orc

        x = g.integers(-act, act, size=(n, d), dtype=np.int64)
        w = g.integers(-(1 << 15), 1 << 15, size=(d, h), dtype=np.int64)
        t0 = time.perf_counter()
        orc.linear_witness(x, w, None, sc)
        t1 = time.perf_counter()
        orc.block_witness(bx, bw, bel, bgl, bcfg)
        t2 = time.perf_counter()
        cpu = {"fc_ms": round((t1 - t0) * 1e3, 1), "block_ms": round((t2 - t1) * 1e3, 1),
               "cores": 1, "kind": "port", "cpu": _cpu_model()}
    print(json.dumps({"mode": "witness", "config": "gpt2_31", "steps": args.steps,
                      "timing": "host wall clock per call", "layers": out,
                      "forward_linear_device_ms": round(forward, 3),
                      "block_witness_host_arrays_ms": block_ms, "cpu_oracle": cpu}),
          flush=True)


def main() -> None:
    global LOG_M, LOG_N, MU
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch-serve", action="store_true",
                    help="line mode: leave out the batched and served measurements")
    ap.add_argument("--overlap", action="store_true",
                    help="timeline mode: a fresh commit before every prove (as in the step)")
    ap.add_argument("--connections", type=int, default=0,
                    help="CUDA_DEVICE_MAX_CONNECTIONS for this process (0: the driver default)")
    ap.add_argument("--mode", choices=["line", "batch", "serve", "commit", "timeline", "basefold",
                                       "logup", "witness", "sumcheck", "autotune"],
                    default="line")
    ap.add_argument("--log-m", type=int, default=LOG_M)
    ap.add_argument("--log-n", type=int, default=LOG_N)
    ap.add_argument("--lanes", type=int, default=12)
    ap.add_argument("--engine", action="store_true",
                    help="autotune mode: also tune the engine lanes on the batch workload")
    ap.add_argument("--mus", default="20,22,24", help="sumcheck mode: polynomial sizes")
    ap.add_argument("--sc-d", type=int, default=3, choices=[1, 2, 3],
                    help="sumcheck mode: factors in the product (the reference bench: 3)")
    ap.add_argument("--shapes", default="10x10,12x12,13x13",
                    help="commit mode: comma-separated log_m x log_n shapes")
    ap.add_argument("--mu", type=int, default=None, help="logup mode: one shape, 2^mu queries")
    ap.add_argument("--nu", type=int, default=16, help="logup mode: 2^nu table entries")
    ap.add_argument("--requests", type=int, default=600)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--layer", default=None,
                    choices=["qkv", "attn_proj", "fc", "fproj", "vocab_head"],
                    help="witness mode: time this linear layer only (no block, no oracle)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.connections:
        os.environ["CUDA_DEVICE_MAX_CONNECTIONS"] = str(args.connections)  # before CUDA starts
    LOG_M, LOG_N, MU = args.log_m, args.log_n, args.log_m + args.log_n
    if args.mode == "batch":
        run_batch(args)
        return
    if args.mode == "serve":
        run_serve(args)
        return
    if args.mode == "commit":
        run_commit(args)
        return
    if args.mode == "timeline":
        run_timeline(args)
        return
    if args.mode == "basefold":
        run_basefold(args)
        return
    if args.mode == "logup":
        run_logup(args)
        return
    if args.mode == "witness":
        run_witness(args)
        return
    if args.mode == "sumcheck":
        run_sumcheck(args)
        return
    if args.mode == "autotune":
        run_autotune(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
