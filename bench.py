"""Benchmark of the graph-construction hot path (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload: one synthetic assembly at binning scale — 100 genomes, 50,000 large
contigs (~420 Mbp), S = 20 coverage samples, --sketch-m 500, --max-edges 200
(the reference's fused N > 25000 path with the mutual filter and the
abundance-first prune).  A step is one full pass of the hot path over it:
2-bit packing, canonical 4-mer counting + GC-norm weights, ProbMinHash
registers, b0, unit rank rows, all-pairs compare with per-row top-200, the
calibration, the mutual filter and the edge weights.  Metric: contig pairs
scored per second, N(N-1)/2 per step per assembly.

* ``value``: inputs resident in HBM when the timed region starts (ASCII
  sequences + coverage, 420 MB > 126 MB L2, so no flush is needed).
* ``e2e``: the same step through the public C ABI call ``rbg_bin_graph`` with
  host buffers: pinned host -> device copies of the inputs and the device ->
  host read of the edge arrays inside the timed region.
* multi-GPU: each rank processes its own assembly of the same size (weak
  scaling over independent assemblies, no collective on the data path).
* ``--impl reference``: RabbitBin's own CPU code (oracle/_ref, compiled from
  the reference sources) on a bounded sample of the same workload with all
  host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(workload="binning-scale assembly: 100 genomes, 50000 contigs, S=20, "
                         "sketch-m 500, max-edges 200, fused path + mutual filter",
                n_genomes=100, n_contigs=50000, samples=20, sketch_m=500, max_edges=200,
                inputs_exceed_l2=True, seed=1)
METRIC = "contig-pairs scored/s"
UNIT = "pairs/s"
# INT32 lanes per SM assumed for the integer peak of the all-pairs roofline
# (SMs x lanes x sampled SM clock); the measured peaks carry no INT32 figure.
INT32_LANES_PER_SM = 128
# DRAM bytes (read + write) and integer ALU pipe share of the symmetric
# all-pairs pass on the default workload (50,000 contigs, S = 20): its two
# kernels, the tcgen05 prefilter and the per-block check and compare, one
# launch each, from one ncu capture of the timed step:
#   ncu --clock-control none -k regex:"k_sym_prefilter|k_sym_check" -s 2 -c 2 --metrics
#     gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum,
#     sm__pipe_alu_cycles_active.avg.pct_of_peak_sustained_active
#     python bench.py --steps 1 --warmup 1 --no-cpu-baseline --no-e2e
# (prefilter 0.627 ms, 6.50 + 4.74 MB, ALU 53.8%; check 1.051 ms, 132.0 + 155.7 MB,
# ALU 50.7%; the ALU share below is their time-weighted mean).  Reported only
# when the timed workload is that one.
ALLPAIRS_NCU = {"contigs": 50000, "samples": 20,
                "dram_bytes": 12854016 + 4613632 + 131647232 + 155896576,
                "alu_pipe_frac": (0.460032 * 0.4908 + 1.020576 * 0.5053) / (0.460032 + 1.020576)}


class ClockSampler:
    """SM clocks and throttle reasons sampled every 5 ms during a timed region
    (NVML reads only; nvidia-smi at 50 ms when NVML is unavailable)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index, period_s=0.005):
        self.index, self.period, self.rows, self.proc, self.nvml = index, period_s, [], None, None
        self.mx = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.nvml, self.h, self.stop = pynvml, h, threading.Event()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nvml = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _poll(self):
        nv = self.nvml
        while not self.stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.rows.append((sm, rs))
            except Exception:
                pass
            self.stop.wait(self.period)

    def _read(self):
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            try:
                rs = sum(bit for (name, bit), v in zip(
                    [("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
                     ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4)], r[5:9])
                    if v.lower() == "active")
                self.mx = float(r[2])
                self.rows.append((float(r[1]), rs))
            except (ValueError, IndexError):
                pass

    def __exit__(self, *a):
        if self.nvml is not None:
            self.stop.set()
            self.t.join(timeout=2)
            return
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [r[0] for r in self.rows]
        reasons = sorted({n for _, rs in self.rows for n, b in self.REASONS.items() if rs & b})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.mx,
                "reasons": reasons, "samples": len(sm),
                "sampler": "nvml 5 ms" if self.nvml is not None else "nvidia-smi 50 ms"}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


LARGE = dict(workload="large single assembly: 300 genomes, 300000 contigs, S=30 with 10% of "
                       "genomes absent per sample, sketch-m 500, max-edges 200, fused path",
             n_genomes=300, n_contigs=300000, samples=30, sketch_m=500, max_edges=200,
             inputs_exceed_l2=True, seed=3, absent_frac=0.1)


def _assembly(seed):
    from rabbitbin_b200.synth import make_assembly
    w = WORKLOAD
    return make_assembly(w["n_genomes"], w["n_contigs"], w["samples"], seed=seed,
                         absent_frac=w.get("absent_frac", 0.0))


def _apply_size(args):
    """--contigs/--samples shrink the workload (profiling cases only)."""
    if args.contigs:
        WORKLOAD["n_contigs"] = args.contigs
        WORKLOAD["workload"] = (f"reduced assembly for profiling: {WORKLOAD['n_genomes']} genomes, "
                                f"{args.contigs} contigs, S={args.samples or WORKLOAD['samples']}")
    if args.samples:
        WORKLOAD["samples"] = args.samples


def run_b200(args):
    import torch
    from rabbitbin_b200 import api

    from rabbitbin_b200 import shard
    rank, world, local = shard.env_rank()
    shard.init(world, "nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    asm = _assembly(shard.shard_seed(WORKLOAD["seed"], rank))
    buf, offs = asm.concat()
    n = asm.n
    pairs = n * (n - 1) // 2
    params = api.default_params(m=WORKLOAD["sketch_m"], max_edges=WORKLOAD["max_edges"])
    ctx = api.Context(local)

    def barrier():
        shard.barrier(world)
        torch.cuda.synchronize(dev)

    # ── device-resident value ───────────────────────────────────────────────
    ctx.stage(buf, offs, asm.depth)
    for _ in range(args.warmup):
        ctx.run_resident(params)
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    timings = []
    barrier()
    with ClockSampler(local) as clk:
        start.record(ext)
        for _ in range(args.steps):
            timings.append(ctx.run_resident(params))
        end.record(ext)
        barrier()
    ms = shard.max_over_ranks(start.elapsed_time(end) / args.steps, world, dev)
    value = shard.whole_job_rate(pairs, world, ms / 1000.0)

    # ── end to end through rbg_bin_graph with pinned host inputs ────────────
    e2e_ms, e2e_edges, e2e_clk = float("nan"), 0, None
    if not args.no_e2e:
        e2e_ms, e2e_edges, e2e_clk = _e2e(args, ctx, buf, offs, asm, params, barrier, world, dev)
    result_e2e = None if args.no_e2e else {
        "value": world * pairs / (e2e_ms / 1000.0), "unit": UNIT, "ms_per_step": e2e_ms,
        "h2d_bytes_per_step": int(len(buf) + offs.nbytes + asm.depth.nbytes),
        "d2h_bytes_per_step": int(e2e_edges * 16),
        "time": "host clock around the rbg_bin_graph calls (each returns with its edges on "
                "the host), barrier before and after, max over ranks",
        "clocks": e2e_clk}
    last = timings[-1]
    return _finish(args, ctx, asm, timings, last, ms, value, result_e2e, clk, world, rank, dev)


def _e2e(args, ctx, buf, offs, asm, params, barrier, world, dev):
    import torch
    pin_seq = torch.empty(len(buf), dtype=torch.uint8, pin_memory=True)
    pin_seq.numpy()[:] = np.frombuffer(buf, dtype=np.uint8)
    pin_depth = torch.empty(asm.depth.shape, dtype=torch.float32, pin_memory=True)
    pin_depth.numpy()[:] = asm.depth
    seq_ptr = pin_seq.numpy().ctypes.data_as(__import__("ctypes").c_char_p)
    # warm-up as for the resident loop; each result stays alive until the next
    # call returns, as in the timed loop, so the result pool holds two blocks
    g = None
    for _ in range(max(args.warmup, 2)):
        g = ctx.bin_graph(seq_ptr, offs, pin_depth.numpy(), params)
    del g
    barrier()
    e2e_edges = 0
    with ClockSampler(int(dev.index or 0)) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            g = ctx.bin_graph(seq_ptr, offs, pin_depth.numpy(), params)
            e2e_edges = len(g["src"])
        barrier()
        wall = time.perf_counter() - t0
    from rabbitbin_b200 import shard
    e2e_ms = shard.max_over_ranks(wall * 1000.0 / args.steps, world, dev)
    return e2e_ms, e2e_edges, clk.summary()


def _finish(args, ctx, asm, timings, last, ms, value, result_e2e, clk, world, rank, dev):
    import torch
    peaks, peak_src = _peaks()
    clocks = clk.summary()
    n, S, m = asm.n, WORKLOAD["samples"], WORKLOAD["sketch_m"]
    mpad = (m + 15) // 16 * 16
    ap_ms = last["allpairs_ms"]
    sym = last["pairs_prefiltered"] > 0
    # dominant kernel: the all-pairs pass.  Its algorithmic work is the register
    # compare of every pair that reaches it: ceil(m/4) packed 32-bit word
    # compares of 8-bit register codes per pair, against the INT32 issue rate
    # of the SMs at the clock sampled during the timed region.
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    sm_mhz = clocks["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)
    int_peak = sms * INT32_LANES_PER_SM * sm_mhz * 1e6 / 1e9          # Gop/s
    pairs_u = n * (n - 1) / 2.0
    p_pmh = last["pairs_compared"] if sym else 2.0 * pairs_u
    words = -(-m // 4)
    int_ach = p_pmh * words / (ap_ms / 1000.0) / 1e9 if ap_ms > 0 else 0.0
    # secondary: the FP16 tensor-core prefilter of the symmetric pass (2 S FLOPs
    # per unordered pair)
    tc_ach = 2.0 * S * pairs_u / (ap_ms / 1000.0) / 1e12 if ap_ms > 0 and sym else 0.0
    tc_peak = peaks.get("bf16_tflops", 1590.0)
    ncu_match = (n == ALLPAIRS_NCU["contigs"] and S == ALLPAIRS_NCU["samples"] and sym)
    traffic = ALLPAIRS_NCU["dram_bytes"] if ncu_match else None
    # sketch: ASCII read, 2-bit words + invalid mask written and read back,
    # per-contig 1/w rows written and read, two code rows written
    nbases = sum(len(q) for q in asm.seqs)
    sk_ms = last["pack_ms"] + last["count_ms"] + last["sketch_ms"]
    sk_bytes = nbases * (1.0 + 3.0 / 8.0 + 3.0 / 8.0) + n * (136 * 8 * 2 + 2 * mpad)
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8/u32 register codes, f64 sketch, f32 abundance",
        "data": "synthetic (seeded order-3 Markov genomes, lognormal coverage)",
        "config": dict(WORKLOAD, parallelism=f"{world} independent assemblies"),
        "e2e": result_e2e,
        "stages_ms": {k: round(v, 4) for k, v in last.items() if k.endswith("_ms")},
        "pairs_prefiltered": last["pairs_prefiltered"],
        "pairs_compared": last["pairs_compared"],
        "pairs_counted": "unordered (symmetric pass)" if sym else "ordered",
        "gpu_launches": int(last["kernel_launches"]) * args.steps,
        "roofline": {
            "bound": "int32",
            "kernel": ("k_sym_prefilter + k_sym_check (tcgen05 FP16 prefilter, exact check and "
                       "register compare of the survivors, each unordered pair once)" if sym else
                       "dense regime: one-hot int8 contraction + row top-K"),
            "achieved": int_ach, "peak": int_peak, "unit": "Gop/s",
            "frac": int_ach / int_peak if int_peak else None,
            "work": f"P_pmh x ceil(m/4) packed 32-bit register compares per launch "
                    f"(P_pmh = {int(p_pmh)} pairs reaching the compare)",
            "peak_source": f"{sms} SMs x {INT32_LANES_PER_SM} INT32 lanes x {sm_mhz:.0f} MHz "
                           "(median SM clock sampled in the timed region; the measured peaks "
                           "carry no INT32 figure)",
            "time": "CUDA events around the all-pairs launch on its stream, last timed step",
            "traffic": traffic,
            "alu_pipe_frac_ncu": ALLPAIRS_NCU["alu_pipe_frac"] if ncu_match else None,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                              "of each kernel of the pass on this workload" if ncu_match else None,
            "secondary": {"bound": "tensor", "what": "FP16 prefilter, 2 S FLOPs per unordered pair",
                          "achieved": tc_ach, "peak": tc_peak, "unit": "TFLOP/s",
                          "frac": tc_ach / tc_peak if tc_peak else None,
                          "peak_source": ("bf16_tflops of MEASURED_PEAKS.json" if peak_src == "measured"
                                          else "fallback 1590 TFLOP/s (MEASURED_PEAKS.json absent)")}},
        "sketch": {"contigs_per_s": n / (sk_ms / 1000.0) if sk_ms > 0 else 0.0,
                   "ms": sk_ms, "bytes": sk_bytes,
                   "achieved_gbs": sk_bytes / (sk_ms / 1000.0) / 1e9 if sk_ms > 0 else 0.0,
                   "hbm_peak_gbs": peaks.get("hbm_gbs", 6650.0),
                   "frac_hbm": (sk_bytes / (sk_ms / 1000.0) / 1e9) / peaks.get("hbm_gbs", 6650.0)
                   if sk_ms > 0 else 0.0,
                   "peak_source": ("hbm_gbs of MEASURED_PEAKS.json" if peak_src == "measured"
                                   else "fallback 6650 GB/s (MEASURED_PEAKS.json absent)")},
        "clocks": clocks,
    }
    ref_graph = None
    if rank == 0 and not args.no_cpu_baseline:
        result["cpu_baseline"], ref_graph = cpu_baseline(asm, seconds=args.cpu_seconds)
    if rank == 0 and (ref_graph is not None or args.check):
        result["parity"] = parity(ctx.fetch_graph(), asm, ref_graph)
    ctx.close()
    from rabbitbin_b200 import shard
    shard.finish(world)
    if rank == 0:
        print(json.dumps(result))


def _ref_lib():
    import oracle
    lib = oracle.ref()
    if lib is None:
        return oracle.restated(), "port"
    return lib, "reference"


def cpu_baseline(asm, seconds=20.0):
    """RabbitBin's own CPU code on a bounded sample of the workload (the first
    50,000 contigs: the whole default workload).  Returns the baseline record
    and, when the sample is the whole workload, the reference's graph."""
    import oracle
    lib, kind = _ref_lib()
    cores = os.cpu_count() or 1
    n = min(asm.n, 50000)
    buf, offs = asm.concat()
    sub_offs = offs[:n + 1]
    t0 = time.perf_counter()
    w = lib.build_winners(buf[:int(sub_offs[-1])], sub_offs, nthreads=cores)
    p = oracle.default_params(n, 500, asm.n_samples, force_path=2, nthreads=cores)
    g = lib.run_graph(p, w, asm.depth[:n])
    dt = time.perf_counter() - t0
    pairs = n * (n - 1) // 2
    return ({"value": pairs / dt, "unit": UNIT, "cores": cores, "kind": kind,
             "sample": f"{n} contigs of the workload (sketch + fused graph + weights), "
                       f"one pass, {dt:.1f} s"},
            g if n == asm.n else None)


def parity(got, asm, ref_graph=None):
    """The timed workload's device graph against RabbitBin's own code on the
    same inputs (run here when not given): edge set, sComp, weights, b0 and
    cutoff identical; the weights' largest distance to the FP64 recomputation."""
    import oracle
    lib, kind = _ref_lib()
    t0 = time.perf_counter()
    if ref_graph is None:
        buf, offs = asm.concat()
        w = lib.build_winners(buf, offs)
        ref_graph = lib.run_graph(oracle.default_params(asm.n, WORKLOAD["sketch_m"],
                                                        asm.n_samples), w, asm.depth)
    ref_s = time.perf_counter() - t0
    s, d, sc, sw = oracle.sorted_edges(ref_graph)
    order = np.lexsort((got["dst"], got["src"]))
    same = (got["b0"] == ref_graph["b0"] and got["sim_cutoff"] == ref_graph["sim_cutoff"] and
            len(order) == len(s) and
            all(np.array_equal(np.asarray(got[k])[order], v)
                for k, v in (("src", s), ("dst", d), ("scomp", sc), ("score", sw))))
    rep = oracle.fp64_report(asm.depth, got)
    return {"config": WORKLOAD["workload"], "against": f"{kind} ({'oracle/_ref' if kind == 'reference' else 'oracle port'})",
            "identical": bool(same), "edges": int(len(order)), "b0": got["b0"],
            "sim_cutoff": got["sim_cutoff"], "max_abs_err_fp64": rep["max_abs_err_fp64"],
            "fp64_cut_disagreements": rep["cut_disagreements"],
            "fp64_max_margin_disagreeing": rep["max_margin_disagreeing"],
            "reference_s": round(ref_s, 2)}


def run_shard_form(args):
    """Strong scaling: ONE assembly split by rows over the ranks
    (rbg_bin_graph_sharded; sketch rows, row maxima and neighbour lists cross
    NVLink through an NCCL allgather of device buffers).  Each step is a full
    call on this rank's contigs from pinned host memory; the time is the
    slowest rank's, and the rate counts the assembly's pairs once."""
    import ctypes
    import torch
    from rabbitbin_b200 import api, shard
    rank, world, local = shard.env_rank()
    shard.init(world, "nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    asm = _assembly(WORKLOAD["seed"])            # the same assembly on every rank
    buf, offs = asm.concat()
    n = asm.n
    pairs = n * (n - 1) // 2
    lo, hi = shard.row_range(n, rank, world)
    local_bytes = np.frombuffer(buf[offs[lo]:offs[hi]], dtype=np.uint8)
    pin_seq = torch.empty(len(local_bytes), dtype=torch.uint8, pin_memory=True)
    pin_seq.numpy()[:] = local_bytes
    seq_ptr = pin_seq.numpy().ctypes.data_as(ctypes.c_char_p)
    local_offs = offs[lo:hi + 1] - offs[lo]
    pin_depth = torch.empty((hi - lo, asm.depth.shape[1]), dtype=torch.float32, pin_memory=True)
    pin_depth.numpy()[:] = asm.depth[lo:hi]
    params = api.default_params(m=WORKLOAD["sketch_m"], max_edges=WORKLOAD["max_edges"])
    ctx = api.Context(local)
    if world > 1:
        gather, devbuf = shard.device_allgather(), True
    else:
        gather, devbuf = (lambda s, r, nb: ctypes.memmove(r, s, nb)), False

    def step():
        return ctx.bin_graph_sharded(seq_ptr, local_offs, pin_depth.numpy(), rank, world, gather,
                                     device_buffers=devbuf, params=params)
    g = None
    for _ in range(max(args.warmup, 2)):
        g = step()
    del g
    shard.barrier(world)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    edges = 0
    for _ in range(args.steps):
        g = step()
        edges = len(g["src"])
    shard.barrier(world)
    ms = shard.max_over_ranks((time.perf_counter() - t0) * 1000.0 / args.steps, world, dev)
    result = {
        "metric": METRIC, "value": pairs / (ms / 1000.0), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "u8/u32 register codes, f64 sketch, f32 abundance",
        "data": "synthetic (seeded order-3 Markov genomes, lognormal coverage)",
        "config": dict(WORKLOAD, parallelism=f"one assembly in {world} row shards"),
        "e2e": {"value": pairs / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms,
                "h2d_bytes_per_step": int(len(local_bytes) + local_offs.nbytes + pin_depth.numpy().nbytes),
                "d2h_bytes_per_step": int(edges * 16)},
        "note": "host inputs to host edges on every rank (the sharded call has no resident form)",
    }
    ctx.close()
    shard.finish(world)
    if rank == 0:
        print(json.dumps(result))


def run_reference(args):
    from rabbitbin_b200 import shard
    rank, world, _ = shard.env_rank()
    if rank != 0:
        return
    import oracle
    lib = oracle.ref()
    kind = "reference"
    if lib is None:
        lib, kind = oracle.restated(), "port"
    asm = _assembly(WORKLOAD["seed"])
    cores = os.cpu_count() or 1
    n = min(asm.n, args.ref_contigs)
    buf, offs = asm.concat()
    sub_offs = offs[:n + 1]
    sbuf = buf[:int(sub_offs[-1])]

    def step():
        w = lib.build_winners(sbuf, sub_offs, nthreads=cores)
        p = oracle.default_params(n, 500, asm.n_samples, force_path=2, nthreads=cores)
        lib.run_graph(p, w, asm.depth[:n])

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    ms = (time.perf_counter() - t0) * 1000.0 / args.steps
    pairs = n * (n - 1) // 2
    value = pairs / (ms / 1000.0)
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "impl": "reference",
        "dtype": "u16 winners, f64 sketch, f32 abundance", "data": "synthetic",
        "config": dict(WORKLOAD, reference_sample_contigs=n),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"first {n} contigs of the workload per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def _pin(buf):
    """A pinned host copy of `buf` (bytes) and a char* to it."""
    import ctypes
    import torch
    t = torch.empty(max(len(buf), 1), dtype=torch.uint8, pin_memory=True)
    if len(buf):
        t.numpy()[:len(buf)] = np.frombuffer(buf, dtype=np.uint8)
    return t, t.numpy().ctypes.data_as(ctypes.c_char_p)


def _same_graph(a, b):
    return (a["b0"] == b["b0"] and a["sim_cutoff"] == b["sim_cutoff"] and
            all(np.array_equal(a[k], b[k]) for k in ("src", "dst", "scomp", "score")))


def run_batch_form(args):
    """Batching form: a mixed stream of assemblies in one rbg_bin_batch call per
    step, against the plain form (one rbg_bin_graph call per assembly) on the
    same pinned host inputs; outputs are checked identical."""
    import torch
    from rabbitbin_b200 import api
    from rabbitbin_b200.workloads import iter_stream
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    keep, ent, items = [], [], []
    for it in iter_stream(args.batch_size, seed=2):
        buf, offs = it.asm.concat()
        it.asm.seqs = []                                   # keep only the pinned copy
        pin, ptr = _pin(buf)
        del buf
        keep.append(pin)
        items.append(it)
        ent.append((ptr, offs, it.asm.depth, api.default_params(m=it.m, max_edges=200)))
    gen_s = time.perf_counter() - t0
    ctx = api.Context(0)
    contigs = sum(len(e[1]) - 1 for e in ent)
    pairs = sum((len(e[1]) - 1) * (len(e[1]) - 2) // 2 for e in ent)
    # both forms are warmed on the whole stream (tables, buffer sizes, tile
    # choices) and hand each call's graphs back before the next call
    got = None
    for _ in range(max(args.warmup, 1)):
        got = None
        got, st = ctx.bin_batch(ent)
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            got = None
            got, st = ctx.bin_batch(ent)
        batch_s = (time.perf_counter() - t0) / args.steps
    for e in ent:
        ctx.bin_graph(*e)                                  # warm the plain path
    t0 = time.perf_counter()
    for e in ent:
        ctx.bin_graph(*e)
    plain_s = time.perf_counter() - t0
    identical = all(_same_graph(g, ctx.bin_graph(*e)) for g, e in zip(got, ent))
    res = {
        "metric": "contigs/s (mixed assembly stream, batched)", "value": contigs / batch_s,
        "unit": "contigs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": batch_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/u32 register codes, f64 sketch, f32 abundance",
        "data": "synthetic (seeded order-3 Markov genomes, lognormal coverage)",
        "config": {"workload": f"mixed stream: {len(ent)} assemblies, contigs log-uniform "
                               "[1e3, 1e5], S in {3,5,10,30}, sketch-m in {250,500,1000}, "
                               "max-edges 200", "assemblies": len(ent), "contigs": contigs,
                   "pairs": pairs, "bases": int(sum(len(k) for k in keep)),
                   "inputs": "pinned host memory, copies inside the timed call"},
        "plain": {"value": contigs / plain_s, "ms_per_step": plain_s * 1e3,
                  "calls": len(ent)},
        "speedup_vs_plain": plain_s / batch_s,
        "pairs_per_s": pairs / batch_s, "graphs_per_s": len(ent) / batch_s,
        "outputs_identical": bool(identical),
        "batch_stats": st, "generate_s": gen_s, "clocks": clk.summary(),
    }
    ctx.close()
    print(json.dumps(res))


def _digest(g):
    import hashlib
    h = hashlib.blake2b(digest_size=16)
    for k in ("src", "dst", "scomp", "score"):
        h.update(np.ascontiguousarray(g[k]).tobytes())
    h.update(np.float64([g["b0"], g["sim_cutoff"]]).tobytes())
    return h.hexdigest()


def _serve_trace(srv, pool, trace, warm):
    """Replay an arrival trace [(t_s, pool index)] open-loop; per-request
    (latency stats, digest) in trace order, and the time of the last result."""
    import threading
    for i in warm:                                    # tables, graphs, buffers
        b, o, d, p = pool[i]
        srv.wait(srv.submit(b, o, d, p), timeout=900.0)
    ids = [None] * len(trace)
    t0 = time.perf_counter()

    def submitter():
        for k, (t, i) in enumerate(trace):
            dt = t0 + t - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            b, o, d, p = pool[i]
            ids[k] = srv.submit(b, o, d, p)

    th = threading.Thread(target=submitter)
    th.start()
    out = []
    for k in range(len(trace)):
        while ids[k] is None:
            time.sleep(0.001)
        g, st = srv.wait(ids[k], timeout=900.0)
        out.append((st, _digest(g)))
    th.join()
    return out, time.perf_counter() - t0


def run_serve_form(args):
    """Serving form: an open-loop Poisson stream of assemblies at a stated rate
    through the request loop (rbg_server, requests folded into shared launches),
    and the same trace through the plain per-request path."""
    import torch
    from rabbitbin_b200 import api
    from rabbitbin_b200.workloads import iter_stream
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    pool, keep, sizes = [], [], []
    for it in iter_stream(args.pool, seed=4, n_min=500, n_max=200000,
                          s_choices=tuple(range(3, 31)), m_choices=(250, 500, 1000)):
        buf, offs = it.asm.concat()
        sizes.append(it.n)
        it.asm.seqs = []
        pin, ptr = _pin(buf)
        del buf
        keep.append(pin)
        pool.append((ptr, offs, it.asm.depth, api.default_params(m=it.m, max_edges=200)))
    gen_s = time.perf_counter() - t0
    rng = np.random.default_rng(4)
    trace, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / args.rate))
        if t >= args.duration:
            break
        trace.append((t, int(rng.integers(0, len(pool)))))
    warm = [int(np.argmin(sizes)), int(np.argmax(sizes))]
    modes = {}
    for mode in args.serve_modes.split(","):
        srv = api.Server(workers=1 if mode == "plain" else args.workers, plain=(mode == "plain"),
                         hbm_budget=150 << 30, max_batch=64)
        with ClockSampler(0) as clk:
            res, wall = _serve_trace(srv, pool, trace, warm)
        srv.close()
        lat = np.array([st["latency_ms"] for st, _ in res])
        contigs = sum(sizes[i] for _, i in trace)
        # server-side span: first submit to last result of the trace
        span = max(st["done_s"] for st, _ in res) - min(st["submit_s"] for st, _ in res)
        modes[mode] = {
            "graphs_per_s": len(trace) / span, "contigs_per_s": contigs / span,
            "span_s": span,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p999_ms": float(np.percentile(lat, 99.9)), "mean_ms": float(lat.mean()),
            "mean_queue_ms": float(np.mean([st["queue_ms"] for st, _ in res])),
            "mean_service_ms": float(np.mean([st["service_ms"] for st, _ in res])),
            "mean_batch": float(np.mean([st["batch_size"] for st, _ in res])),
            "max_batch": int(max(st["batch_size"] for st, _ in res)),
            "wall_s": wall, "clocks": clk.summary(), "digests": [d for _, d in res]}
    identical = (modes["batched"]["digests"] == modes["plain"]["digests"]
                 if len(modes) == 2 else None)
    for m in modes.values():
        m.pop("digests")
    b = modes.get("batched") or modes["plain"]
    pl = modes.get("plain") or b
    res = {
        "metric": f"served graphs/s (Poisson {args.rate:g} req/s)", "value": b["graphs_per_s"],
        "unit": "graphs/s", "n_gpus": 1, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/u32 register codes, f64 sketch, f32 abundance",
        "data": "synthetic (seeded order-3 Markov genomes, lognormal coverage)",
        "config": {"workload": f"open-loop Poisson arrivals at {args.rate:g} req/s for "
                               f"{args.duration:g} s; assemblies from a pool of {len(pool)} drawn "
                               "with contigs log-uniform [500, 2e5], S in 3..30, sketch-m in "
                               "{250,500,1000}, max-edges 200; HBM budget 150 GB",
                   "workers": args.workers,
                   "requests": len(trace), "pool_contigs": sizes,
                   "inputs": "pinned host memory, copies inside each request"},
        "latency_ms": {"p50": b["p50_ms"], "p99": b["p99_ms"], "p999": b["p999_ms"]},
        "batched": modes.get("batched"), "plain": modes.get("plain"),
        "graphs_per_s_vs_plain": b["graphs_per_s"] / pl["graphs_per_s"],
        "outputs_identical": identical, "generate_s": gen_s,
    }
    print(json.dumps(res))


def run_lpa_form(args):
    """Label propagation (the step after the graph): the Fisher sweep on the
    binning-scale graph, device-resident and through the host-buffer C-ABI call,
    against the reference's own cluster_by_propagation on the host cores
    (identical labels checked)."""
    import torch
    from rabbitbin_b200 import api
    torch.cuda.set_device(0)
    asm = _assembly(WORKLOAD["seed"])
    buf, offs = asm.concat()
    n = asm.n
    params = api.default_params(m=WORKLOAD["sketch_m"], max_edges=WORKLOAD["max_edges"])
    ctx = api.Context(0)
    g = ctx.bin_graph(buf, offs, asm.depth, params)
    src, dst, score = (np.array(g[k]) for k in ("src", "dst", "score"))
    out = {}
    for sync in (False, True):
        for _ in range(max(args.warmup, 1)):
            ctx.label_propagation_resident(n, seed=1, rule="fisher", synchronous=sync)
        with ClockSampler(0) as clk:
            t0 = time.perf_counter()
            dev = []
            for _ in range(args.steps):
                lab, st = ctx.label_propagation_resident(n, seed=1, rule="fisher",
                                                         synchronous=sync)
                dev.append(st["incidence_ms"] + st["sweep_ms"])
            wall = (time.perf_counter() - t0) * 1000.0 / args.steps
        t0 = time.perf_counter()
        for _ in range(args.steps):
            lab_h, _ = ctx.label_propagation(n, src, dst, score, seed=1, rule="fisher",
                                             synchronous=sync)
        e2e = (time.perf_counter() - t0) * 1000.0 / args.steps
        out["sync" if sync else "gs"] = dict(
            device_ms=float(np.median(dev)), resident_call_ms=wall, e2e_ms=e2e,
            rounds=st["rounds"], changes=st["changes"], frozen=st["frozen"], arcs=st["arcs"],
            incidence_ms=st["incidence_ms"], sweep_ms=st["sweep_ms"], labels=int(len(np.unique(lab))),
            clocks=clk.summary(), _lab=lab, _lab_h=lab_h)
    ref = None
    if not args.no_cpu_baseline:
        import oracle
        R = oracle.ref()
        if R is not None:
            ref = {}
            for key in ("gs", "sync"):
                if key == "sync":
                    os.environ["RABBIT_PAR_LPA"] = "1"
                t0 = time.perf_counter()
                want = R.label_propagation(n, src, dst, score, seed=1, nthreads=os.cpu_count())
                ref[key] = dict(ms=(time.perf_counter() - t0) * 1000.0,
                                identical=bool((want == out[key]["_lab"]).all() and
                                               (want == out[key]["_lab_h"]).all()))
                os.environ.pop("RABBIT_PAR_LPA", None)
    for v in out.values():
        v.pop("_lab")
        v.pop("_lab_h")
    gs = out["gs"]
    res = {
        "metric": "label propagation time per graph (Fisher, sequential sweep)",
        "value": gs["device_ms"], "unit": "ms", "n_gpus": 1, "higher_is_better": False,
        "form": "lpa", "steps": args.steps, "warmup": args.warmup,
        "config": {"workload": WORKLOAD["workload"] + "; its graph, then label propagation",
                   "nodes": n, "edges": int(len(src)), "seed": 1},
        "e2e": {"value": gs["e2e_ms"], "unit": "ms",
                "h2d_bytes_per_step": int(len(src) * 12), "d2h_bytes_per_step": int(n * 4)},
        "sweeps": out,
        "cpu_baseline": None if ref is None else {
            "kind": "reference", "cores": os.cpu_count(), "value": ref["gs"]["ms"], "unit": "ms",
            "sample": "the whole graph (the sequential sweep uses one thread; the synchronous "
                      "one all cores)", "sweeps": ref},
    }
    print(json.dumps(res))


def run_depth_form(args):
    """BAM -> depth (the step before the path when the bin command gets BAMs):
    one (--bams: several) coordinate-sorted BAM(s) of 150 bp reads over the binning-scale assembly
    (seeded synthetic reads, mean depth 2x, htslib-style BGZF at deflate level
    6) through rbg_bam_depth_mem: BGZF bytes in host memory in, the depth
    matrix back in host memory.  Checked against the reference's own
    depth_accumulate_sample on the same records; its per-read pass on the host
    cores (records already decoded, so without its BGZF decoding) is the CPU
    baseline."""
    import torch
    from rabbitbin_b200 import api
    from rabbitbin_b200.synth import BAM_CLEAN, bam_records, make_bam
    torch.cuda.set_device(0)
    asm = _assembly(WORKLOAD["seed"])
    buf, offs = asm.concat()
    lens = np.diff(offs).astype(np.uint32)
    nbam = max(1, args.bams)
    t0 = time.perf_counter()
    bams = []
    for b in range(nbam):
        # one BAM per coverage sample of the assembly, mean depth 2x
        cov = np.asarray(asm.depth[:, b % asm.depth.shape[1]], np.float64)
        cov = cov * (2.0 / max(cov.mean(), 1e-9))
        bams.append(make_bam(lens, cov, names=[f"contig_{i}" for i in range(asm.n)], seq=buf,
                             seq_off=offs, seed=7 + b, read_len=150, level=6, **BAM_CLEAN))
    bam_bytes = sum(len(x) for x in bams)
    gen_s = time.perf_counter() - t0
    ctx = api.Context(0)
    for _ in range(max(args.warmup, 1)):
        out = ctx.bam_depth(bams)
    walls, kern, infl = [], [], []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            t1 = time.perf_counter()
            out = ctx.bam_depth(bams)
            walls.append((time.perf_counter() - t1) * 1000.0)
            kern.append(out["kernel_ms"])
            infl.append(out["inflate_ms"])
    ms = float(np.median(walls))
    recs = out["records"]
    ub = out["decompressed_bytes"]
    kms = float(np.median(kern))
    # per-record algorithmic bytes of k_depth_reads: the fixed fields (36), the
    # CIGAR (4 per op) and the aux fields it walks, plus its 4-byte offset; the
    # records' sequence, quality and name bytes are never read
    pk = _peaks()[0]
    res = {
        "metric": "BAM records summarised/s (reads into per-contig depth)",
        "value": recs / (ms / 1000.0), "unit": "records/s", "n_gpus": 1, "higher_is_better": True,
        "form": "depth", "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "dtype": "u8 records, u64 sums, f32 means", "data": "synthetic (seeded reads over the "
        "binning-scale assembly's contigs)",
        "config": {"workload": "BAM -> depth: 50,000-contig binning-scale assembly, "
                   f"{nbam} BAM(s) of 150 bp reads ({recs} in all; mean depth 2x each), "
                   "BGZF level 6", "bams": nbam,
                   "records": recs, "bam_bytes": bam_bytes, "decompressed_bytes": ub,
                   "generation_s": round(gen_s, 2), "inputs_exceed_l2": True},
        "e2e": {"value": recs / (ms / 1000.0), "unit": "records/s",
                "h2d_bytes_per_step": int(ub), "d2h_bytes_per_step": int(out["means"].nbytes +
                                                                         out["sums"].nbytes),
                "time": "host clock around rbg_bam_depth_mem (BGZF bytes in host memory in, the "
                        "depth matrix in host memory out)"},
        "stages_ms": {"host_prefix_ms": float(np.median(infl)), "kernel_ms": kms,
                      "call_ms": float(out["total_ms"]), "total_ms": ms},
        "decompressed_gbs": ub / (ms / 1000.0) / 1e9,
        "device_route": bool(out["device_bams"] == nbam),
        "kernels": {"names": "k_inflate + k_walk (2 passes) + k_scan_counts + k_depth_reads_dev "
                             "per chunk, k_depth_means per call",
                    "device_ms": kms, "records_per_s": recs / (kms / 1000.0),
                    "inflated_gbs": ub / (kms / 1000.0) / 1e9},
        # k_inflate is 96% of the route's device time (launch list of this
        # workload); its algorithmic bytes are the compressed blocks read and
        # the inflated bytes written
        "roofline": {"bound": "hbm", "kernel": "k_inflate (with walk and rule: 96% inflate)",
                     "achieved": (bam_bytes + ub) / (kms / 1000.0) / 1e9,
                     "peak": pk.get("hbm_gbs") if pk else 6650.0, "unit": "GB/s",
                     "frac": (bam_bytes + ub) / (kms / 1000.0) / 1e9 /
                             (pk.get("hbm_gbs") if pk else 6650.0),
                     "peak_source": "hbm_gbs of MEASURED_PEAKS.json" if pk else "fallback",
                     "traffic": 1.85 * (bam_bytes + ub),
                     "traffic_source": "ncu dram__bytes_read+write of k_inflate on the 8,000-contig "
                                       "case (1.85x its algorithmic bytes: the CRC pass re-reads "
                                       "the output), scaled by bytes",
                     "note": "latency-bound Huffman decode chain, not bandwidth"},
        "gpu_launches": 5 * sum(max(1, -(-(ub // nbam) // (1024 << 20))) for _ in range(nbam)) + 1,
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        import oracle
        if oracle.ref_depth() is not None:
            ref_s, sums_ok, means_ok, avgs = 0.0, True, True, []
            for b, bam in enumerate(bams):
                raw, tl, _ = bam_records(bam)
                t0 = time.perf_counter()
                want, avg = oracle.depth_accumulate_ref(raw, tl, 0.97, 75, False, 0,
                                                        threads=os.cpu_count() or 1)
                ref_s += time.perf_counter() - t0
                means = oracle.depth_means(want, tl, min(75, avg // 3))
                sums_ok &= bool(np.array_equal(out["sums"][b], want))
                means_ok &= bool(np.array_equal(out["means"][:, b], means[out["tid"]]))
                avgs.append(avg)
            res["cpu_baseline"] = {
                "kind": "reference", "cores": os.cpu_count(), "value": recs / ref_s,
                "unit": "records/s", "sample": "every BAM's records, already decoded "
                "(depth_accumulate_sample: its BGZF decoding is not timed)",
                "ms": ref_s * 1000.0}
            res["parity"] = {"against": "reference (oracle/_ref)", "avg_read": avgs,
                             "sums_identical": sums_ok, "means_identical": means_ok}
    print(json.dumps(res))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ref-contigs", type=int, default=50000)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--check", action="store_true",
                    help="compare the device graph with the reference's on the whole workload "
                         "(always done when the CPU baseline covers the whole workload)")
    ap.add_argument("--serve-modes", default="batched,plain",
                    help="serve form: which request loops replay the trace")
    ap.add_argument("--contigs", type=int, default=0, help="profiling: fewer contigs")
    ap.add_argument("--samples", type=int, default=0, help="profiling: other S")
    ap.add_argument("--form", default="plain", choices=["plain", "batch", "serve", "lpa", "depth"],
                    help="plain: the binning-scale assembly; batch: a mixed stream per call; "
                         "serve: a Poisson request stream through the request loop; lpa: label "
                         "propagation on the binning-scale graph; depth: BAM -> depth over "
                         "the binning-scale assembly")
    ap.add_argument("--batch-size", type=int, default=64, help="batch form: assemblies")
    ap.add_argument("--bams", type=int, default=1, help="depth form: BAMs per call")
    ap.add_argument("--config", default="binning", choices=["binning", "large"],
                    help="binning: 50,000 contigs, S=20 (default); large: 300,000 contigs, S=30")
    ap.add_argument("--rate", type=float, default=20.0, help="serve form: requests per second")
    ap.add_argument("--duration", type=float, default=10.0, help="serve form: seconds of arrivals")
    ap.add_argument("--pool", type=int, default=32, help="serve form: distinct assemblies")
    ap.add_argument("--workers", type=int, default=0,
                    help="serve form: lanes (0: the server's default of two, one taking "
                         "large requests first, one small requests only)")
    ap.add_argument("--shard", default="assemblies", choices=["assemblies", "rows"],
                    help="multi-GPU: one assembly per rank (weak scaling, default) or one "
                         "assembly split by rows over the ranks (strong scaling)")
    args = ap.parse_args()
    if args.config == "large":
        WORKLOAD.clear()
        WORKLOAD.update(LARGE)
    _apply_size(args)
    if args.impl == "reference":
        run_reference(args)
    elif args.form == "batch":
        run_batch_form(args)
    elif args.form == "serve":
        run_serve_form(args)
    elif args.form == "lpa":
        run_lpa_form(args)
    elif args.form == "depth":
        run_depth_form(args)
    elif args.shard == "rows":
        run_shard_form(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
