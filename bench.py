"""Throughput of the Mars exhaustive domain-range search on B200.

One step = the exhaustive search of every RD-quadtree node of one 512x512 synthetic
grayscale plane (block sizes 32, 16, 8 and 4, domain stride 2, 8 isometries) -- the search
work of one encode at the 512x512 exhaustive configuration (seeds 1-8, cycled).  The metric
is range x domain x isometry fits per second, with evals counted exactly as the reference
counts them (domain positions x 8 per node).

  value : device time of one step with the planes already in HBM: a search plan's CUDA
          graph (contraction + every level's statistics, seed, correlation and finish
          kernels) launched once per step, CUDA events on the launching stream around it;
          L2 flushed between steps by a 256 MiB write.
  e2e   : the same work through the public call a caller makes per plane,
          mars_search_plan_run: host plane in (through pinned staging), the full node
          table back on the host, timed on the host around the synchronous call; the
          one-shot factory mars_search_table_build is reported beside it.
  cpu_baseline : the CPU oracle (a C++ restatement of the reference's CPU search) on a
          bounded sample of the same nodes, all host threads.

`--impl reference` times the reference algorithm on the host cores instead (the oracle
port: the reference's own Rust cannot be built in this image).
Multi-GPU: one process per GPU (torchrun); each rank searches its own planes (weak
scaling, no collective on the data path); value = all ranks' fits / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mars_b200 import synthetic  # noqa: E402

W = H = 512
SIZES = (32, 16, 8, 4)
SHIFT = 2
METRIC = "range·domain·isometry fits/s (512² exhaustive)"
UNIT = "fits/s"
WORKLOAD = ("exhaustive search of every RD quadtree node of a 512x512 synthetic gray plane, "
            "block sizes 32..4, domain stride 2, 8 isometries, seeds 1-8")


# Figures that only ncu measures (bench.py cannot run under a profiler), copied from the
# committed captures named beside them; re-captured whenever the kernel changes.
# DRAM bytes (read + write) per launch of the dominant search kernel, s=4 level.
NCU_SOURCE = "profiles/corr_tc_s4_512x512_ncu.md"
NCU_TRAFFIC = {4: 21_360_000}
# DRAM bytes (read + write) of one all-levels correlation launch (corr_tc_all_kernel, every
# level of one 512x512 plane): profiles/corr_tc_all_512x512_ncu.md.
NCU_ALL_SOURCE = "profiles/corr_tc_all_512x512_ncu.md"
NCU_ALL_TRAFFIC = 42_626_816 + 299_264
# Thread instructions per candidate fit of the correlation kernel's level (warp
# instructions x 32 / fits, same capture): the issue cost behind the epilogue roofline.
NCU_INSTR_PER_FIT = {4: 0.8684e9 * 32 / 8.52e9, 8: 0.3886e9 * 32 / 2.0e9}
# DRAM bytes of one decode iteration, by plane side (profiles/decode_cell_4096x4096_ncu.md;
# profiles/decode_sorted_16384x16384_ncu.md: dram__bytes.sum.per_second x
# gpu__time_duration.sum of the gather and the place launch of one iteration).
NCU_DECODE_TRAFFIC = {4096: 34_831_104 + 748_800, 16384: 651_660_000 + 802_090_000}
# The kernels of one decode iteration: the cell kernel while the two planes total at most
# 96 MiB, the source-ordered gather and place beyond (api.cu, want_sorted_decode).
DECODE_SORTED_BYTES = 96 << 20


def rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_seeds(rank):
    """The 8 planes a rank cycles through: seeds 1-8, rank r starting at seed r % 8 + 1."""
    return [1 + (rank + k) % 8 for k in range(8)]


def reduce_max(value, dist=None, device=None):
    """Max of a per-rank float over all ranks (the identity without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def level_nodes(size):
    rows, cols = np.meshgrid(np.arange(H // size) * size, np.arange(W // size) * size, indexing="ij")
    return rows.ravel().astype(np.uint32), cols.ravel().astype(np.uint32)


def level_evals(size, shift=SHIFT):
    nd = ((H - 2 * size) // shift + 1) * ((W - 2 * size) // shift + 1)
    return nd * 8


def evals_per_step():
    return sum(level_evals(s) * (H // s) * (W // s) for s in SIZES)


def macs_of_level(size):
    return level_evals(size) * (H // size) * (W // size) * size * size


class ClockSampler:
    """SM clock and throttle reasons sampled every few ms through NVML during the timed
    region (nvidia-smi every 200 ms as a fallback)."""
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap"}

    def __init__(self, device):
        self.device = device
        self.samples = []  # (sm_mhz, max_mhz, reason bits)
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device)
        except Exception:
            self._nvml = None

    def _sample_nvml(self):
        n = self._nvml
        sm = n.nvmlDeviceGetClockInfo(self._h, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(self._h, n.NVML_CLOCK_SM)
        try:
            bits = n.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        except Exception:
            bits = n.nvmlDeviceGetCurrentClocksThrottleReasons(self._h)
        return (float(sm), float(mx), int(bits))

    def _sample_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                              "--format=csv,noheader,nounits"], capture_output=True, text=True,
                             timeout=5).stdout.strip().split(",")
        bits = 0
        for b, f in zip((0x8, 0x40, 0x20, 0x4), out[2:6]):
            bits |= b if f.strip().lower() == "active" else 0
        return (float(out[0]), float(out[1]), bits)

    def _run(self):
        period = 0.005 if self._nvml else 0.2
        while not self._stop.is_set():
            try:
                self.samples.append(self._sample_nvml() if self._nvml else self._sample_smi())
            except Exception:
                pass
            self._stop.wait(period)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [x[0] for x in self.samples]
        reasons = sorted({name for x in self.samples for bit, name in self.REASONS.items()
                          if x[2] & bit})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(x[1] for x in self.samples),
                "reasons": reasons, "samples": len(self.samples),
                "source": "nvml" if self._nvml else "nvidia-smi"}


def cpu_sample_blocks(cores):
    """Blocks per level of the CPU sample: 8 per host thread (every thread busy through the
    oracle's one-block dynamic schedule), capped at the level's node count.  The GPU line's
    cpu_baseline and the reference arm use this same sample."""
    return {s: min(len(level_nodes(s)[0]), 8 * cores) for s in SIZES}


def cpu_baseline(seed=1, single_core=True):
    """The oracle (reference CPU search restated in C++) on a fixed random sample of the
    step's nodes per level, all host threads.  Returns (fits/s over the full step's eval
    mix, cores, description, single-core ns per eval or None, measured sample seconds)."""
    from oracle import oracle as orc
    img = synthetic.gray(W, H, seed)
    p = orc.make_params(min_size=4, max_size=32, shift=SHIFT)
    cores = os.cpu_count() or 1
    counts = cpu_sample_blocks(cores)
    total_time = sample_s = 0.0
    for size in SIZES:
        rows, cols = level_nodes(size)
        pick = np.random.default_rng(size).permutation(len(rows))[:counts[size]]
        t0 = time.perf_counter()
        orc.search_blocks(img, size, SHIFT, p, rows[pick], cols[pick], nthreads=0)
        el = time.perf_counter() - t0
        sample_s += el
        rate = len(pick) * level_evals(size) / el
        total_time += level_evals(size) * len(rows) / rate
    value = evals_per_step() / total_time
    ns_per_eval = None
    if single_core:
        # One host thread on the s=8 level's first nodes, for the per-eval cost of one core.
        rows, cols = level_nodes(8)
        t0 = time.perf_counter()
        orc.search_blocks(img, 8, SHIFT, p, rows[:8], cols[:8], nthreads=1)
        ns_per_eval = (time.perf_counter() - t0) / (8 * level_evals(8)) * 1e9
    desc = ("oracle search_blocks (one block per OpenMP work item) on a fixed random sample of "
            "the 512x512 seed-1 step's nodes per level "
            f"({', '.join(f's{s}: {n} blocks' for s, n in counts.items())}), {cores} threads; "
            "per-level fits/s combined over the full step's eval mix")
    return value, cores, desc, ns_per_eval, sample_s


DECODE_SIDE = 4096         # the decode GB/s figure: both planes (2 x 16.8 MB) fit in L2
DECODE_SIDE_LARGE = 16384  # both planes (2 x 268 MB) exceed L2: the HBM-resident case
DECODE_ITERS = 10


def decode_header(mb, side):
    """Header of the synthetic decode map: encmars defaults (bits 4/7, sizes 4..32, stride 2,
    max_alfa 1.0 -> int_max_alfa 32)."""
    return mb.Header(bits_alfa=4, bits_beta=7, min_size=4, max_size=32, shift=2, width=side,
                     height=side, int_max_alfa=32)


def decode_cpu_baseline(side=2048, seed=1):
    """The oracle's decode_iterative (single-threaded, as the reference's) on a smaller
    plane of the same synthetic map."""
    from oracle import oracle as orc
    leaves = synthetic.quadtree_leaves(side, side, seed)
    hdr = orc.Header(bits_alfa=4, bits_beta=7, min_size=4, max_size=32, shift=2, width=side,
                     height=side, int_max_alfa=32)
    t0 = time.perf_counter()
    orc.decode(hdr, leaves, DECODE_ITERS)
    el = time.perf_counter() - t0
    return {"value": side * side * DECODE_ITERS / el, "unit": "pixel-iterations/s", "cores": 1,
            "kind": "port",
            "sample": f"oracle decode of a {side}x{side} synthetic quadtree map, "
                      f"{DECODE_ITERS} iterations"}


def run_decode(args, mb, ctx, stream, dev, peaks, side, with_cpu, flush=None):
    """Fixed-point decode: DECODE_ITERS iterations of the gather over a synthetic quadtree
    map of a side x side plane, from the flat-128 seed.  `flush` (a device buffer larger
    than L2) is rewritten between timed decodes when the planes would otherwise stay in L2."""
    import torch
    leaves = synthetic.quadtree_leaves(side, side, 1)
    hdr = decode_header(mb, side)
    plan = ctx.decode_plan(hdr, leaves)
    out = torch.empty(side * side, dtype=torch.uint8, device=dev)
    for _ in range(max(3, args.warmup)):
        plan.run(DECODE_ITERS, out.data_ptr())
    torch.cuda.synchronize(dev)
    steps = max(3, min(args.steps, 10))
    launches0 = ctx.launches
    t = 0.0
    with ClockSampler(dev.index) as clocks:
        for k in range(steps):
            if flush is not None:
                flush.fill_(k & 0xFF)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.run(DECODE_ITERS, out.data_ptr())
            e1.record(stream)
            torch.cuda.synchronize(dev)
            t += e0.elapsed_time(e1) / 1e3
    launches = ctx.launches - launches0
    plan.close()
    t_dec = t / steps
    px = side * side
    algo = DECODE_ITERS * (2 * px + 16 * len(leaves))
    achieved = algo / t_dec / 1e9
    try:
        peak, src = float(peaks["hbm_gbs"]), "measured copy bandwidth"
    except Exception:
        peak, src = 6650.0, "fallback 6.65 TB/s"
    # End to end through mars_decode: host leaves in, host image out.
    t0 = time.perf_counter()
    ctx.decode(hdr, leaves, DECODE_ITERS)
    t_e2e = time.perf_counter() - t0
    del out
    resident = 2 * px < 126e6
    return {
        "workload": f"decode_iterative of a {side}x{side} synthetic quadtree map "
                    f"({len(leaves)} leaves, sizes 32..4, modes 0/1/2), {DECODE_ITERS} iterations "
                    "from the flat-128 seed",
        "value": px * DECODE_ITERS / t_dec, "unit": "pixel-iterations/s",
        "ms_per_decode": 1e3 * t_dec, "steps": steps, "gpu_launches": launches,
        "l2": ("planes L2-resident across the iterations of one decode; L2 flushed between "
               "timed decodes (256 MiB write)") if resident else
              "not flushed: both planes exceed L2",
        "clocks": clocks.summary(),
        "roofline": {"bound": "hbm",
                     "kernel": ("sorted_gather_kernel + sorted_place_kernel"
                                if 2 * px > DECODE_SORTED_BYTES else "decode_cell_kernel"),
                     "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": NCU_DECODE_TRAFFIC.get(side), "peak_source": src,
                     "bytes_per_launch": algo / DECODE_ITERS,
                     "launch_ms": 1e3 * t_dec / DECODE_ITERS},
        "e2e": {"value": px * DECODE_ITERS / t_e2e, "unit": "pixel-iterations/s",
                "h2d_bytes_per_step": len(leaves) * 44, "d2h_bytes_per_step": px},
        "cpu_baseline": decode_cpu_baseline() if with_cpu else None,
    }


REFINE_SEEDS = tuple(range(1, 9))
REFINE_LAMBDAS = (50.0, 100.0, 200.0, 400.0, 800.0)
REFINE_STEPS = 20
REFINE_DECODE_ITERS = 12
REFINE_DOMAIN_PASSES = 5
REFINE_ROUNDS = 1


def run_refine(mb, ctx, stream, dev, peaks, seeds=REFINE_SEEDS, lambdas=REFINE_LAMBDAS,
               domain_passes=REFINE_DOMAIN_PASSES, rounds=REFINE_ROUNDS):
    """Attractor refinement at 512x512: per seed 1-8 and lambda 50..800, the GPU RD encode
    (modes 0-3, block sizes 32..4, domain stride 2), the domain re-search against the
    attractor (`domain_passes` passes of mars_refine_domains) and the (s, o) refinement of the
    result (20 steps); PSNR-Y of the exact 12-iteration decodes against the bytes of the
    .mars streams.  `domain_only_bd_psnr_db` is the gain of the re-search alone.  The gain is the
    BD-PSNR of the refined curve over the plain one per seed (PCHIP in log bpp over the
    overlap, the reference's mars-bench BD contract: 5 points per curve), averaged over
    seeds; the per-lambda gains at the same lambda are listed beside it (the byte counts of
    a plain stream and its refinement differ by well under 1 %)."""
    import torch
    from mars_b200 import rd

    def psnr(a, b):
        mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
        return 10.0 * np.log10(255.0 ** 2 / mse)

    per_seed, gains, enc_t, ref_t, dom_t, accepted = [], {l: [] for l in lambdas}, [], [], [], 0
    bytes_ratio, dom_bd = [], []
    for seed in seeds:
        img = synthetic.gray(W, H, seed)
        plain, refined, domain_only = [], [], []
        for lam in lambdas:
            params = mb.make_params(min_size=4, max_size=32, shift=SHIFT, lam=lam)
            t0 = time.perf_counter()
            hdr, leaves, res, _ = ctx.encode(img, params, allowed_modes=(1, 1, 1, 1))
            enc_t.append(time.perf_counter() - t0)
            b0 = len(mb.format_write(hdr, leaves, res))
            t0 = time.perf_counter()
            start = leaves
            if domain_passes:
                start, _ = ctx.refine_domains(params, hdr, leaves, img, res,
                                              passes=domain_passes,
                                              decode_iterations=REFINE_DECODE_ITERS)
            dom_t.append(time.perf_counter() - t0)
            plan = ctx.refine_plan(hdr, start, img, res)
            out, rep = plan.run(steps=REFINE_STEPS, lr=1.0, decode_iterations=REFINE_DECODE_ITERS)
            plan.close()
            for _ in range(rounds - 1):
                # Further rounds: domains re-searched against the refined attractor, then
                # (s, o) again; each step keeps its input when it does not decode better.
                nxt, _ = ctx.refine_domains(params, hdr, out, img, res, passes=domain_passes,
                                            decode_iterations=REFINE_DECODE_ITERS)
                plan = ctx.refine_plan(hdr, nxt, img, res)
                out, rep2 = plan.run(steps=REFINE_STEPS, lr=1.0,
                                     decode_iterations=REFINE_DECODE_ITERS)
                plan.close()
            ref_t.append(time.perf_counter() - t0)
            accepted += int(rep.accepted or any(start != leaves))
            b1 = len(mb.format_write(hdr, out, res))
            bd_ = len(mb.format_write(hdr, start, res))
            p0 = psnr(ctx.decode(hdr, leaves, REFINE_DECODE_ITERS, res), img)
            p1 = psnr(ctx.decode(hdr, out, REFINE_DECODE_ITERS, res), img)
            pd = psnr(ctx.decode(hdr, start, REFINE_DECODE_ITERS, res), img)
            plain.append((rd.bpp(b0, W, H), p0))
            refined.append((rd.bpp(b1, W, H), p1))
            domain_only.append((rd.bpp(bd_, W, H), pd))
            gains[lam].append(p1 - p0)
            bytes_ratio.append(b1 / b0)
        if len(lambdas) >= rd.MIN_POINTS_PER_CURVE:
            r = rd.bd_metrics(plain, refined, ("plain", "refined"))
            per_seed.append({"seed": seed, "bd_psnr_db": r.bd_psnr_db,
                             "bd_rate_pct": r.bd_rate_pct, "bpp_interval": r.bd_psnr_bpp_interval,
                             "plain": plain, "refined": refined})
            if domain_passes:
                dom_bd.append(rd.bd_metrics(plain, domain_only, ("plain", "domains")).bd_psnr_db)
    # BD metrics need at least 4 points per curve; shorter sweeps report per-lambda gains only.
    bd = float(np.mean([p["bd_psnr_db"] for p in per_seed])) if per_seed else None

    # Per-iteration cost of the two solves on one plan (fixed iteration counts).
    img = synthetic.gray(W, H, 1)
    hdr, leaves, res, _ = ctx.encode(img, mb.make_params(min_size=4, max_size=32, shift=SHIFT,
                                                         lam=200.0), allowed_modes=(1, 1, 1, 1))
    plan = ctx.refine_plan(hdr, leaves, img, res)
    s0, o0 = plan.params()
    iters = 256
    plan.forward(s0, o0, max_iters=8, tol=0.0)
    plan.backward(max_iters=8, tol=0.0)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    plan.forward(s0, o0, max_iters=iters, tol=0.0)
    t_fwd = (time.perf_counter() - t0) / iters
    t0 = time.perf_counter()
    plan.backward(max_iters=iters, tol=0.0)
    t_adj = (time.perf_counter() - t0) / iters
    plan.close()
    return {
        "workload": "attractor refinement of the GPU RD encode, 512x512 synthetic gray, seeds "
                    "1-8, lambda 50/100/200/400/800, modes 0-3, sizes 32..4, domain stride 2; "
                    f"{rounds} round(s) of {domain_passes} domain re-search passes, then "
                    f"{REFINE_STEPS} (s, o) steps; "
                    f"exact decodes of {REFINE_DECODE_ITERS} iterations",
        "metric": "PSNR-Y gain at equal bytes (BD-PSNR, refined vs plain GPU search)",
        "value": bd, "unit": "dB", "higher_is_better": True,
        "domain_passes": domain_passes, "rounds": rounds,
        "domain_only_bd_psnr_db": float(np.mean(dom_bd)) if dom_bd else None,
        "ms_per_domain_refine": 1e3 * float(np.median(dom_t)),
        "per_lambda_gain_db": {str(int(l)): float(np.mean(g)) for l, g in gains.items()},
        "bytes_ratio_refined_over_plain": [float(min(bytes_ratio)), float(max(bytes_ratio))],
        "accepted": f"{accepted}/{len(seeds) * len(lambdas)}",
        "per_seed": [{k: v for k, v in p.items() if k in ("seed", "bd_psnr_db", "bd_rate_pct")}
                     for p in per_seed],
        "ms_per_refine": 1e3 * float(np.median(ref_t)),
        "encode": {"value": 1.0 / float(np.median(enc_t)), "unit": "images/s",
                   "note": "ctx.encode (search, walks and mode pricing; from a geometry's "
                           "second encode on through the context's search plan) of one "
                           "512x512 plane, host buffers in and leaves out, median over the "
                           f"{len(enc_t)} encodes above"},
        "us_per_forward_iter": 1e6 * t_fwd, "us_per_adjoint_iter": 1e6 * t_adj,
        "note": "the 512x512 refinement iterates on L2-resident f32 planes (1 MiB each): "
                "launch- and latency-bound, so its cost is quoted per iteration, not as GB/s",
    }


def run_encode(mb, ctx, workers=3):
    """Whole RD encodes of the 512x512 planes (seeds 1-8, lambda 200, sizes 32..4, stride 2):
    the search on the GPU and the host walks, host plane in, leaves out.  `value`: images/s
    through Context.encode_many (a search plan per size, `workers` planes in flight so one
    plane's walks overlap the next one's search); `sequential`: one ctx.encode after
    another; `planned_sequential`: one planned encode after another (search, warm-up walk,
    pricing and RD walk on the device; the host builds the rate snapshot and receives the
    leaves).  Both for the default modes {0, 2} and for all four modes: the four-mode encode
    prices every quadtree node (the residual mode's DCTs) on the device, the two-mode one on
    the host walk."""
    imgs = [synthetic.gray(W, H, s) for s in range(1, 9)]
    params = mb.make_params(min_size=4, max_size=32, shift=SHIFT, lam=200.0)
    out = {"workload": "RD encode (search + walks + mode pricing) of 8 synthetic 512x512 gray "
                       "planes, lambda 200, sizes 32..4, domain stride 2",
           "unit": "images/s", "workers": workers,
           "pricing": {"modes_0_2": "host walk", "modes_0_3": "device (rdprice.cu), one warp "
                       "per quadtree node"}}
    for key, modes in (("modes_0_2", (1, 0, 1, 0)), ("modes_0_3", (1, 1, 1, 1))):
        ctx.encode_many(imgs[:2], params, workers=workers, allowed_modes=modes)
        t0 = time.perf_counter()
        ctx.encode_many(imgs, params, workers=workers, allowed_modes=modes)
        piped = len(imgs) / (time.perf_counter() - t0)
        for _ in range(2):  # a geometry's second encode makes the context's plan for it
            ctx.encode(imgs[0], params, allowed_modes=modes)
        t0 = time.perf_counter()
        for im in imgs:
            ctx.encode(im, params, allowed_modes=modes)
        seq = len(imgs) / (time.perf_counter() - t0)
        plan = ctx.cached_plan(W, H, params)
        plan.encode(imgs[0], allowed_modes=modes)
        t0 = time.perf_counter()
        for im in imgs:
            plan.encode(im, allowed_modes=modes)
        planned = len(imgs) / (time.perf_counter() - t0)
        out[key] = {"value": piped, "sequential": seq, "planned_sequential": planned}
    out["value"] = out["modes_0_2"]["value"]
    return out


CLASSIFIED_SEEDS = (1, 2, 3, 4)


def run_classified(mb, ctx):
    """Classified search on 768x512 colour: synthetic RGB (the generator per channel, random
    3x3 channel mix), BT.601 YCbCr with Cb/Cr box-downsampled to 4:2:0 on the device, then
    the Fisher-classified search (domains bucketed by the reference's block classification)
    of every RD-quadtree node of the three planes, ranges 16..4, domain stride 2.  `value`:
    classified fits/s over the planes of seeds 1-4 (host planes in, node tables out, the
    colour conversion included); `exhaustive` the same planes through the exhaustive search;
    `encode` whole colour RD encodes (lambda 200, all modes, Fisher) into MARC bytes."""
    from mars_b200 import color
    rgbs = [synthetic.rgb(768, 512, s) for s in CLASSIFIED_SEEDS]
    params = mb.make_params(min_size=4, max_size=16, shift=SHIFT, lam=200.0)

    def planes(rgb):
        y, cb, cr = ctx.ycbcr(rgb[..., 0], rgb[..., 1], rgb[..., 2])
        return [y, ctx.downsample_box(cb), ctx.downsample_box(cr)]

    def searched(method):
        ev = 0
        t0 = time.perf_counter()
        for rgb in rgbs:
            for pl in planes(rgb):
                prov = ctx.search_provider(pl, params, method=method)
                ev += int(mb.lib().mars_search_table_evals(prov._h))
                prov.close()
        return ev, time.perf_counter() - t0

    # One graph-captured Fisher plan per plane geometry (Y and the two chroma planes), made
    # before the timed loop, as a caller encoding many images of one size keeps them.
    plans = {}
    for pl in planes(rgbs[0]):
        if pl.shape not in plans:
            plans[pl.shape] = ctx.search_plan(pl.shape[1], pl.shape[0], params, method="fisher")

    def planned():
        ev = 0
        t0 = time.perf_counter()
        for rgb in rgbs:
            for pl in planes(rgb):
                t = plans[pl.shape].run(pl)
                ev += int(mb.lib().mars_search_table_evals(t._h))
                t.close()
        return ev, time.perf_counter() - t0

    for method in ("fisher", "exhaustive"):  # warm-up
        for pl in planes(rgbs[0]):
            ctx.search_provider(pl, params, method=method).close()
    planned()
    launches0 = ctx.launches
    ev_f, t_f = planned()
    launches = ctx.launches - launches0
    ev_ff, t_ff = searched("fisher")
    ev_x, t_x = searched("exhaustive")
    for plan in plans.values():
        plan.close()
    cparams = color.ColorEncodeParams(params, params, method="fisher")
    # Two untimed encodes: the context makes its search plans on a geometry's second encode.
    color.encode_color(ctx, rgbs[0], cparams)
    color.encode_color(ctx, rgbs[1], cparams)
    nbytes = 0
    t0 = time.perf_counter()
    for rgb in rgbs:
        data, _ = color.encode_color(ctx, rgb, cparams)
        nbytes += len(data)
    t_e = time.perf_counter() - t0
    return {
        "workload": "768x512 synthetic RGB (seeds 1-4, random channel mix) -> YCbCr 4:2:0 "
                    "on the device, Fisher-classified search of every RD quadtree node of Y, "
                    "Cb, Cr (ranges 16..4, domain stride 2)",
        "value": ev_f / t_f, "unit": "fits/s", "evals": ev_f, "seconds": t_f,
        "images_per_s": len(rgbs) / t_f, "gpu_launches": launches,
        "call": "Fisher search plans (mars_indexed_plan_create, one per plane geometry, made "
                "before timing): mars_search_plan_run per plane",
        "factory": {"value": ev_ff / t_ff, "unit": "fits/s", "seconds": t_ff,
                    "images_per_s": len(rgbs) / t_ff,
                    "call": "mars_indexed_table_build per plane (node lists and scratch per "
                            "call)"},
        "exhaustive": {"value": ev_x / t_x, "unit": "fits/s", "evals": ev_x, "seconds": t_x,
                       "images_per_s": len(rgbs) / t_x},
        "encode": {"value": len(rgbs) / t_e, "unit": "colour images/s",
                   "bytes_per_image": nbytes / len(rgbs),
                   "call": "color.encode_color (Fisher, lambda 200, modes 0-3, MARC bytes; "
                           "the context's cached Fisher and exhaustive search plans)"},
        "timing": "host wall clock, host planes in and host tables / bytes out, one image "
                  "after another",
    }


UNEVEN_COUNT, UNEVEN_SEED, UNEVEN_LARGE = 64, 5, 4096


def run_uneven(mb, ctx, dev, large=True):
    """Uneven batch: 64 gray planes with sides drawn (seeded) from {128, 256, 384, 512, 768,
    1024}, then one 4096x4096 plane; every RD-quadtree node of each (sizes 32..4, domain
    stride 2, lambda 200 nodes) searched through the provider factory with host planes in
    and host tables out, one plane after another on one context."""
    import torch
    sides = synthetic.batch_sides(UNEVEN_COUNT, UNEVEN_SEED)
    imgs = [synthetic.gray(s, s, 100 + i) for i, s in enumerate(sides)]
    params = mb.make_params(min_size=4, max_size=32, shift=SHIFT, lam=200.0)
    ctx.search_provider(imgs[0], params).close()
    torch.cuda.synchronize(dev)

    def timed(planes):
        ev = 0
        t0 = time.perf_counter()
        for im in planes:
            prov = ctx.search_provider(im, params)
            ev += int(mb.lib().mars_search_table_evals(prov._h))
            prov.close()
        return ev, time.perf_counter() - t0

    launches0 = ctx.launches
    ev_b, t_b = timed(imgs)
    out = {
        "workload": f"{UNEVEN_COUNT} synthetic gray planes, sides from "
                    "{128,256,384,512,768,1024} (seed 5), exhaustive search of every RD "
                    "quadtree node, sizes 32..4, domain stride 2",
        "value": ev_b / t_b, "unit": "fits/s", "evals": ev_b, "seconds": t_b,
        "images_per_s": len(imgs) / t_b, "gpu_launches": ctx.launches - launches0,
        "timing": "host wall clock around the provider factory (host plane in, node table "
                  "out), planes one after another",
    }
    if large:
        big = synthetic.gray(UNEVEN_LARGE, UNEVEN_LARGE, 99)
        ev_l, t_l = timed([big])
        out["large"] = {"workload": f"one {UNEVEN_LARGE}x{UNEVEN_LARGE} plane, same search",
                        "value": ev_l / t_l, "unit": "fits/s", "evals": ev_l, "seconds": t_l}
    return out


RANKED_K = 3  # candidates per node of the ranked-search leg (rd_candidates)


def run_ranked(mb, ctx, dev):
    """Ranked search (search_candidates, k = RANKED_K): every RD-quadtree node of the 512x512
    planes of the search leg through the ranked provider factory, host plane in and host
    table out, on the tensor-core kernel and (beside it) the CUDA-core kernel."""
    import torch
    params = mb.make_params(min_size=4, max_size=32, shift=SHIFT)
    imgs = [synthetic.gray(W, H, s) for s in (1, 2, 3)]

    def timed(c):
        c.search_provider(imgs[0], params, k=RANKED_K).close()
        torch.cuda.synchronize(dev)
        ev = 0
        t0 = time.perf_counter()
        for im in imgs:
            prov = c.search_provider(im, params, k=RANKED_K)
            ev += int(mb.lib().mars_search_table_evals(prov._h))
            prov.close()
        return ev / (time.perf_counter() - t0)

    tc = timed(ctx)
    simt_ctx = mb.Context(dev.index)
    simt_ctx.set_search_path("simt")
    try:
        simt = timed(simt_ctx)
    finally:
        simt_ctx.close()
    return {"workload": f"ranked search (k = {RANKED_K}) of every RD quadtree node of 512x512 "
                        "synthetic gray planes (seeds 1-3), sizes 32..4, domain stride 2",
            "value": tc, "unit": "fits/s", "cuda_core_value": simt,
            "timing": "host wall clock around the ranked provider factory "
                      "(mars_search_table_build_ranked: host plane in, k-lists out)"}


LARGE_BLOCKS = 1024  # range blocks per level of the large-plane profile case


def run_large_profile(args):
    """The large-plane case of the uneven batch, sized for a profiler: one side x side
    synthetic plane (seed 99), and per level (sizes 32..4, stride 2) the search of its first
    LARGE_BLOCKS aligned range blocks against every domain of the plane through
    mars_search_blocks_device (contraction, domain statistics, operand planes, B operand,
    seeds, correlation, finish; one call per level, CUDA events around the calls).  Prints
    one JSON object: per level the milliseconds per call, the correlation's algorithmic int8
    TOP/s (evals x s^2 MACs x 2) and the algorithmic bytes of its decimation (u8 plane in,
    contracted plane and the level's domain statistics out)."""
    import torch
    import mars_b200 as mb
    side = args.profile_large
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = mb.Context(0)
    ctx.set_stream(stream.cuda_stream)
    plane = torch.from_numpy(synthetic.gray(side, side, 99)).to(dev)
    params = mb.make_params(min_size=4, max_size=32, shift=SHIFT)
    out = {"workload": f"{side}x{side} synthetic gray plane (seed 99): the first {LARGE_BLOCKS} "
                       "aligned range blocks of each level against every domain, stride 2",
           "levels": {}}
    for size in SIZES:
        nb = min(LARGE_BLOCKS, (side // size) ** 2)
        k = np.arange(nb)
        rows = torch.from_numpy(((k // (side // size)) * size).astype(np.int32)).to(dev)
        cols = torch.from_numpy(((k % (side // size)) * size).astype(np.int32)).to(dev)
        res = torch.empty((nb, 80), dtype=torch.uint8, device=dev)

        def call():
            mb.check(mb.lib().mars_search_blocks_device(
                ctx.handle, plane.data_ptr(), side, side, size, SHIFT, mb.C.byref(params),
                rows.data_ptr(), cols.data_ptr(), nb, res.data_ptr()))
        for _ in range(args.warmup):
            call()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            call()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / args.steps
        nd = ((side - 2 * size) // SHIFT + 1) ** 2
        macs = nb * nd * 8 * size * size
        out["levels"][str(size)] = {
            "blocks": nb, "domains": nd, "ms_per_call": ms,
            "int8_tops_algorithmic": 2 * macs / (ms * 1e-3) / 1e12,
            "decimation_bytes": side * side + (side // 2) ** 2 * 4 + nd * 20}
    print(json.dumps({"large_profile": out}), flush=True)
    ctx.close()
    return 0


def run_large_full(args):
    """One whole exhaustive search of a side x side synthetic plane (seed 99): every
    RD-quadtree node, sizes 32..4, stride 2, through mars_search_nodes_device (the levels
    one after another on one stream; plane in HBM, node table left in HBM).  `warmup`
    untimed searches, then one timed with CUDA events.  Prints one JSON object: evals, nodes,
    seconds and fits/s.  At 4096x4096 this is the uneven batch's large plane (4.65e13
    evals, ~17 s per search on one B200), so it is not part of the default run."""
    import torch
    import mars_b200 as mb
    side = args.large_full
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = mb.Context(0)
    ctx.set_stream(stream.cuda_stream)
    plane = torch.from_numpy(synthetic.gray(side, side, 99)).to(dev)
    params = mb.make_params(min_size=4, max_size=32, shift=SHIFT)
    n, ev = mb.C.c_size_t(), mb.C.c_uint64()
    mb.check(mb.lib().mars_search_nodes_device(ctx.handle, plane.data_ptr(), side, side,
                                               mb.C.byref(params), None, 0, mb.C.byref(n),
                                               mb.C.byref(ev)))
    out = torch.empty((n.value, 80), dtype=torch.uint8, device=dev)

    def call():
        mb.check(mb.lib().mars_search_nodes_device(ctx.handle, plane.data_ptr(), side, side,
                                                   mb.C.byref(params), out.data_ptr(), n.value,
                                                   mb.C.byref(n), mb.C.byref(ev)))
    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize(dev)
    with ClockSampler(dev.index) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        call()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    sec = e0.elapsed_time(e1) / 1e3
    print(json.dumps({"large_full": {
        "workload": f"exhaustive search of every RD quadtree node of a {side}x{side} synthetic "
                    "gray plane (seed 99), block sizes 32..4, domain stride 2",
        "nodes": n.value, "evals": ev.value, "seconds": sec, "value": ev.value / sec,
        "unit": "fits/s", "warmup": args.warmup, "clocks": clocks.summary(),
        "call": "mars_search_nodes_device (levels in sequence, no graph)"}}), flush=True)
    ctx.close()
    return 0


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    vals, secs = [], []
    desc, cores = "", os.cpu_count() or 1
    # One warm-up sample at most: every sample is the same few seconds of CPU work.
    for _ in range(min(args.warmup, 1)):
        cpu_baseline(single_core=False)
    for _ in range(args.steps):
        v, cores, desc, _, s = cpu_baseline(single_core=False)
        vals.append(v)
        secs.append(s)
    value = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            # A step here is one bounded sample of the workload (its measured seconds); the
            # full 512x512 step's time is extrapolated from the sample's per-level rates.
            "ms_per_step": 1e3 * float(np.mean(secs)),
            "extrapolated_ms_per_full_step": 1e3 * evals_per_step() / value,
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "i64/f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "image": "512x512", "sizes": list(SIZES),
                       "shift": SHIFT, "evals_per_step": evals_per_step()},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": desc, "sample_seconds": float(np.median(secs))},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference's Rust (cargo) is not installed in this image; its CPU "
                    "search runs as the committed C++ restatement (oracle/), parallelised "
                    "over nodes with OpenMP as the reference does with Rayon"}
    print(json.dumps(line), flush=True)
    return 0


def run_gpu(args):
    import torch
    import mars_b200 as mb

    rank, world, local = rank_info()
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = mb.Context(local)
    # A dedicated stream: the library's kernels and the timing events share it.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    params = mb.make_params(min_size=4, max_size=32, shift=SHIFT)
    seeds = rank_seeds(rank)
    planes = [torch.from_numpy(synthetic.gray(W, H, s)).to(dev) for s in seeds]
    levels = {}
    for size in SIZES:
        r, c = level_nodes(size)
        levels[size] = (torch.from_numpy(r.astype(np.int32)).to(dev),
                        torch.from_numpy(c.astype(np.int32)).to(dev))
    out = {s: torch.empty((len(levels[s][0]), 80), dtype=torch.uint8, device=dev) for s in SIZES}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step(k, timers=None):
        plane = planes[k % len(planes)]
        for size in SIZES:
            rr, cc = levels[size]
            if timers is not None:
                timers[size][0].record(stream)
            mb.check(mb.lib().mars_search_blocks_device(
                ctx.handle, plane.data_ptr(), W, H, size, SHIFT, mb.C.byref(params),
                rr.data_ptr(), cc.data_ptr(), len(rr), out[size].data_ptr()))
            if timers is not None:
                timers[size][1].record(stream)

    # The timed step: every level of one plane as one CUDA-graph launch of a search plan
    # (mars_search_plan_run_device: the plane is copied device to device into the plan's
    # input buffer, then the captured contraction + 4 levels replay).
    plan = ctx.search_plan(W, H, params)
    plan_launches = plan.launches
    ev_step = evals_per_step()
    assert plan.evals == ev_step, (plan.evals, ev_step)
    for k in range(args.warmup):
        plan.run_device(planes[k % len(planes)].data_ptr())
        step(k)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)

    t_graph = 0.0
    t_kernel = 0.0  # the all-levels correlation launch inside each replay (events in the graph)
    kernel_timed = True
    launches0 = ctx.launches
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.fill_(k & 0xFF)  # evict L2 between timed steps (outside the events)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.run_device(planes[k % len(planes)].data_ptr())
            e1.record(stream)
            torch.cuda.synchronize(dev)
            t_graph += e0.elapsed_time(e1) / 1e3
            if kernel_timed:
                try:
                    t_kernel += plan.kernel_ms / 1e3
                except mb.MarsError:  # one launch per level: no all-levels kernel to time
                    kernel_timed = False
    torch.cuda.synchronize(dev)
    launches = ctx.launches - launches0
    t_total = reduce_max(t_graph, dist, dev)
    value = ev_step * args.steps * world / t_total

    # Per-level breakdown (the levels launched one by one, CUDA events around each), which
    # also gives the dominant kernel's launch time for the roofline.
    lvl_steps = max(3, min(args.steps, 10))
    per_level = {s: 0.0 for s in SIZES}
    for k in range(lvl_steps):
        flush.fill_(k & 0xFF)
        timers = {s: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for s in SIZES}
        step(k, timers)
        torch.cuda.synchronize(dev)
        for s in SIZES:
            per_level[s] += timers[s][0].elapsed_time(timers[s][1]) / 1e3

    # The dominant level (the one whose per-level launches take longest) for the epilogue
    # bound; the roofline itself is the all-levels launch when the plan has one.
    dom = max(SIZES, key=lambda s: per_level[s])
    t_launch = per_level[dom] / lvl_steps
    ops = 2.0 * macs_of_level(dom)  # int8-equivalent MAC ops of the correlation
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak_tops = 2.0 * float(peaks["bf16_tflops"])
        peak_src = "2 x measured bf16 dense (int8 dense runs at twice the bf16 rate)"
    except Exception:
        peak_tops = 2.0 * 1590.0
        peak_src = "2 x fallback bf16 1.59 PFLOP/s"
    achieved = ops / t_launch / 1e12
    level_roofline = {"kernel": f"search level s={dom} (one launch per level)",
                      "achieved": achieved, "peak": peak_tops, "unit": "TOP/s",
                      "frac": achieved / peak_tops, "traffic": NCU_TRAFFIC.get(dom),
                      "traffic_source": f"ncu ({NCU_SOURCE})", "ops_per_launch": ops,
                      "launch_ms": 1e3 * t_launch}
    if kernel_timed and t_kernel > 0:
        roof_kernel = "corr_tc_all_kernel: every tensor-core level of the step, one launch"
        roof_ops = 2.0 * sum(macs_of_level(s) for s in SIZES)
        roof_ms = 1e3 * t_kernel / args.steps
        roof_traffic, roof_src = NCU_ALL_TRAFFIC, NCU_ALL_SOURCE
    else:
        roof_kernel = level_roofline["kernel"]
        roof_ops, roof_ms = ops, 1e3 * t_launch
        roof_traffic, roof_src = NCU_TRAFFIC.get(dom), NCU_SOURCE
    roof_achieved = roof_ops / (roof_ms / 1e3) / 1e12
    # The fused epilogue's bound at small s: every candidate costs NCU_INSTR_PER_FIT thread
    # instructions, issued at most one warp instruction per scheduler (4 per SM) per clock.
    epilogue = None
    if dom in NCU_INSTR_PER_FIT:
        props = torch.cuda.get_device_properties(dev)
        clk_mhz = clocks.summary()["sm_mhz"] or 1965.0  # median SM clock of the timed region
        fits_dom = level_evals(dom) * len(level_nodes(dom)[0])
        peak_fits = props.multi_processor_count * 4 * clk_mhz * 1e6 * 32 / NCU_INSTR_PER_FIT[dom]
        epilogue = {"bound": "issue", "kernel": f"search level s={dom}",
                    "achieved": fits_dom / t_launch, "peak": peak_fits, "unit": "fits/s",
                    "frac": fits_dom / t_launch / peak_fits,
                    "instr_per_fit": NCU_INSTR_PER_FIT[dom],
                    "peak_source": f"{props.multi_processor_count} SMs x 4 issue slots x "
                                   f"{clk_mhz:.0f} MHz (sampled median) x 32 threads / thread "
                                   f"instructions per fit ({NCU_SOURCE})"}

    # End to end through the public calls, host plane in and the node table back on the
    # host: the plan's run (what a caller encoding many planes of one size makes per plane)
    # and, beside it, the one-shot provider factory (plan and buffers built per call).
    e2e_val = e2e_factory = None
    h2d = d2h = 0
    host_planes = [synthetic.gray(W, H, s) for s in seeds]
    nodes = sum((H // s) * (W // s) for s in SIZES)
    if rank == 0 or world > 1:
        e2e_steps = max(3, min(args.steps, 10))
        for k in range(min(2, args.warmup)):
            plan.run(host_planes[k % len(host_planes)]).close()
            ctx.search_provider(host_planes[k % len(host_planes)], params).close()
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            plan.run(host_planes[k % len(host_planes)]).close()
        t_e2e = time.perf_counter() - t0
        e2e_val = ev_step * e2e_steps * world / t_e2e
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            ctx.search_provider(host_planes[k % len(host_planes)], params).close()
        e2e_factory = ev_step * e2e_steps * world / (time.perf_counter() - t0)
        h2d = W * H
        d2h = nodes * 80 + 8
    plan.close()

    decode = decode_large = None
    if not args.no_decode:
        with_cpu = rank == 0 and world == 1 and not args.no_cpu
        decode = run_decode(args, mb, ctx, stream, dev, peaks, DECODE_SIDE, with_cpu, flush)
        decode_large = run_decode(args, mb, ctx, stream, dev, peaks, DECODE_SIDE_LARGE, False)

    # The single-GPU legs run at N = 1 only: under torchrun the other ranks would sit in
    # the final barrier for their whole duration.
    single = rank == 0 and world == 1
    encode = run_encode(mb, ctx) if single and not args.no_encode else None

    refine = None
    if single and not args.no_refine:
        refine = run_refine(mb, ctx, stream, dev, peaks)

    uneven = None
    if single and not args.no_uneven:
        uneven = run_uneven(mb, ctx, dev)

    classified = None
    if single and not args.no_classified:
        classified = run_classified(mb, ctx)

    ranked = run_ranked(mb, ctx, dev) if single and not args.no_ranked else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, desc, ns1, secs = cpu_baseline()
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc,
               "sample_seconds": secs, "single_core_ns_per_eval": ns1}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "i32/f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "image": "512x512", "sizes": list(SIZES),
                       "shift": SHIFT, "evals_per_step": ev_step, "nodes_per_step": nodes,
                       "parallelism": f"replicas{world}", "l2": "flushed between steps (256 MiB write)"},
            "roofline": {"bound": "tensor", "kernel": roof_kernel,
                         "achieved": roof_achieved, "peak": peak_tops, "unit": "TOP/s",
                         "frac": roof_achieved / peak_tops, "traffic": roof_traffic,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                           f"({roof_src})",
                         "peak_source": peak_src,
                         "ops_per_launch": roof_ops, "launch_ms": roof_ms,
                         "timing": ("CUDA events recorded inside the plan's graph around the "
                                    "launch (mars_search_plan_kernel_ms), every timed step")
                                   if kernel_timed else "CUDA events around the level's launches",
                         "dominant_level": level_roofline,
                         "epilogue": epilogue},
            "per_level_ms": {str(s): 1e3 * per_level[s] / lvl_steps for s in SIZES},
            "launch": "one CUDA-graph launch per step (search plan), "
                      f"{plan_launches} kernel nodes",
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "call": "mars_search_plan_run",
                    "factory_value": e2e_factory,
                    "factory_call": "mars_search_table_build (node lists and scratch per call)"},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "decode": decode,
            "decode_large": decode_large,
            "encode": encode,
            "refine": refine,
            "uneven": uneven,
            "classified": classified,
            "ranked": ranked,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-decode", action="store_true", help="skip the decode leg")
    ap.add_argument("--no-refine", action="store_true", help="skip the refinement leg")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch leg")
    ap.add_argument("--no-encode", action="store_true", help="skip the RD encode leg")
    ap.add_argument("--no-ranked", action="store_true", help="skip the ranked-search leg")
    ap.add_argument("--no-classified", action="store_true",
                    help="skip the classified colour leg")
    ap.add_argument("--refine-only", action="store_true",
                    help="run only the refinement leg (for profiling), on --refine-seeds and "
                         "--refine-lambdas, and print its JSON object")
    ap.add_argument("--refine-seeds", default=",".join(map(str, REFINE_SEEDS)))
    ap.add_argument("--refine-lambdas", default=",".join(str(int(l)) for l in REFINE_LAMBDAS))
    ap.add_argument("--refine-rounds", type=int, default=REFINE_ROUNDS,
                    help="rounds of (domain re-search, (s, o) refinement)")
    ap.add_argument("--refine-domain-passes", type=int, default=REFINE_DOMAIN_PASSES,
                    help="passes of the domain re-search before the (s, o) refinement")
    ap.add_argument("--decode-only", type=int, default=0, metavar="SIDE",
                    help="run only the decode leg on a SIDE x SIDE synthetic map (for "
                         "profiling) and print its JSON object")
    ap.add_argument("--classified-only", action="store_true",
                    help="run only the classified colour leg (for profiling) and print its "
                         "JSON object")
    ap.add_argument("--profile-large", type=int, default=0, metavar="SIDE",
                    help="run only the large-plane profile case (a SIDE x SIDE plane, the "
                         "first blocks of every level) and print its JSON object")
    ap.add_argument("--large-full", type=int, default=0, metavar="SIDE",
                    help="time one whole exhaustive search of a SIDE x SIDE plane (every RD "
                         "node) and print its JSON object")
    args = ap.parse_args()
    if args.large_full:
        return run_large_full(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_large:
        return run_large_profile(args)
    if args.decode_only:
        import torch
        import mars_b200 as mb
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        stream = torch.cuda.Stream(dev)
        torch.cuda.set_stream(stream)
        ctx = mb.Context(0)
        ctx.set_stream(stream.cuda_stream)
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        print(json.dumps({"decode": run_decode(args, mb, ctx, stream, dev, peaks, args.decode_only,
                                               False)}), flush=True)
        ctx.close()
        return 0
    if args.classified_only:
        import torch
        import mars_b200 as mb
        torch.cuda.set_device(0)
        ctx = mb.Context(0)
        print(json.dumps({"classified": run_classified(mb, ctx)}), flush=True)
        ctx.close()
        return 0
    if args.refine_only:
        import torch
        import mars_b200 as mb
        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        stream = torch.cuda.Stream(dev)
        torch.cuda.set_stream(stream)
        ctx = mb.Context(0)
        ctx.set_stream(stream.cuda_stream)
        out = run_refine(mb, ctx, stream, dev, {},
                         tuple(int(x) for x in args.refine_seeds.split(",")),
                         tuple(float(x) for x in args.refine_lambdas.split(",")),
                         args.refine_domain_passes, args.refine_rounds)
        print(json.dumps({"refine": out}), flush=True)
        ctx.close()
        return 0
    return run_gpu(args)


if __name__ == "__main__":
    raise SystemExit(main())
