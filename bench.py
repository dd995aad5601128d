#!/usr/bin/env python
"""Throughput of racon's polishing hot path on B200: window POA consensus.

Workload (the batched POA + edlib configuration, config 1): seeded
synthetic 1 Mb genome, draft with 1% errors, 50x FASTQ reads (log-normal
8 kb / 4 kb, 12% error, Phred U[5,30]), PAF from true coordinates with +-50 bp
end jitter, racon defaults -w 500 -m 3 -x -5 -g -4 -q 10 -e 0.3. racon's
initialize() (loading, device overlap alignment, layer assembly) runs once,
untimed; a step is the consensus of every window of the job.

  value  windows/s with the windows staged in HBM (rb_poa_run), device time
         from CUDA events on the library's stream, max over ranks
  e2e    windows/s through the C ABI with host buffers, wall time per step:
         the polishing path's own calls (rb_sequences_stage: sequence table
         to the device; rb_poa_stage_overlaps: layers assembled on the
         device from the breaking points; rb_poa_run; rb_poa_fetch)
  e2e_host_layers  the same through rb_poa_batch with host-assembled
         windows (pack every layer's bases, H2D, kernels, D2H, unpack)
  roofline / compute  HBM bytes (bases and qualities in, consensus out) and
         int32 issue of poa_kernel from the edge-cells the kernel counts
         (|layer| x sum_v (1 + in-degree v), 3 int ops each); the POA DP is
         integer-issue bound
  tuning  the launch choices rb_autotune measured on this job
  parity  the oracle's consensus of the CPU sample against the device's,
         window by window
  cpu_baseline  the CPU oracle (restatement of racon's algorithm, not
         reference racon, which does not build here) on a bounded sample of
         the same windows with every host thread
  pipeline  the whole job through rb_polish_files against the oracle's
         pipeline on every host thread, FASTA compared byte for byte
  serving  config-4 jobs through the serving loop (shared consensus and alignment kernels)
         at 80 % of its measured peak

--impl reference runs the CPU oracle as the reference arm (rank 0 only).
Multi-GPU: one process per GPU (torchrun); each rank polishes its own job
(seed + rank), no collective on the data path, weak scaling.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}
# Thread instructions poa_kernel executes per DP cell, from the same kind of
# capture (smsp__inst_executed.sum x threads per instruction / DP cells:
# 6.33 G x 30.19 / 5.84 G)
POA_THREAD_INST_PER_CELL = 6329653471 * 30.19 / 5838774640
# DRAM bytes (read + write) per DP cell of poa_kernel, from one ncu capture of
# config 1 at 0.1 genome scale (1.413 GB read + 14.977 GB written over
# 5.839 G cells); traffic grows with the cells, so a full launch's traffic is
# this times its cells
POA_DRAM_BYTES_PER_CELL = (1.412735e9 + 14.977411e9) / 5838774640
L2_FLUSH_BYTES = 512 << 20
# DRAM bytes (read + write) of nw_distance_kernel per nominal cell (query x
# target span) from one ncu capture of the first 500 pairs of the config-2
# batch (31.4 MB read + 104.8 MB written over 421.3 G nominal cells); the
# strip carry buffers grow with the swept cells
NWD_DRAM_BYTES_PER_CELL = (31.4e6 + 104.8e6) / 421325730898


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--config", type=int, default=1, choices=[0, 1, 2, 3, 4])
    p.add_argument("--scale", type=float, default=1.0, help="genome scale (1.0 = the named workload)")
    p.add_argument("--cpu-sample", type=int, default=400, help="windows in the CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-autotune", action="store_true", help="keep the default launch choices")
    p.add_argument("--no-pipeline", action="store_true", help="skip the whole-job end-to-end comparison")
    p.add_argument("--data-dir", default=None)
    p.add_argument("--serving-jobs", type=int, default=12, help="config-4 jobs in the serving measurement "
                   "(0 = skip it)")
    p.add_argument("--workers", type=int, default=8, help="serving-loop workers")
    p.add_argument("--no-shared-consensus", action="store_true",
                   help="serving: each job launches its own consensus kernel")
    p.add_argument("--no-shared-alignment", action="store_true",
                   help="serving: each job launches its own alignment kernels")
    p.add_argument("--alignment-ctas", type=int, default=0,
                   help="serving: CTAs per SM of the shared alignment kernel (0: 1)")
    p.add_argument("--large-first-every", type=int, default=0,
                   help="serving: every k-th warp of the shared kernels takes the largest jobs first (0: none)")
    p.add_argument("--alignment-yield", type=int, default=0,
                   help="serving: alignment pairs per warp and launch for large jobs (0: persistent)")
    p.add_argument("--alignment-share", type=int, default=0,
                   help="serving: percent of the SMs large jobs' alignment grids fill (0: all)")
    p.add_argument("--pairs", type=int, default=10000, help="config-2 pairs per step")
    return p.parse_args()


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.fh = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.flush()
        self.fh.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.fh.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.fh.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(seconds, world):
    """The largest of every rank's seconds (all ranks call it in the same
    order). The tensor lives where the process group's backend wants it: the
    current CUDA device under NCCL, host memory under gloo."""
    if world <= 1:
        return float(seconds)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_seed(config, rank):
    """Each rank polishes its own job (weak scaling): seed = config + 1000 * rank."""
    return config + 1000 * rank


def _data(args, rank):
    from racon_b200 import synthetic
    base = args.data_dir or os.path.join(tempfile.gettempdir(), "racon_b200_bench")
    d = os.path.join(base, "config%d_scale%g_rank%d" % (args.config, args.scale, rank))
    seed = shard_seed(args.config, rank)
    marker = os.path.join(d, "done")
    if args.config == 3:
        if not os.path.exists(marker):
            r, o, t, info = synthetic.fragment(d, **_fragment_shape(args.scale), seed=seed)
            with open(marker, "w") as fh:
                json.dump(info, fh)
        return os.path.join(d, "reads.fastq"), os.path.join(d, "overlaps.paf"), os.path.join(d, "reads.fastq")
    if not os.path.exists(marker):
        r, o, t, info = synthetic.contig(d, args.config, seed=seed, scale=args.scale)
        with open(marker, "w") as fh:
            json.dump(info, fh)
    ext = "fastq" if args.config == 1 else "fasta"
    return os.path.join(d, "reads." + ext), os.path.join(d, "overlaps.paf"), os.path.join(d, "draft.fasta")


def _fragment_shape(scale):
    """Config 3: 5 Mb truth in 3 contigs, local depth a sinusoid in 10-200x,
    log-normal reads (mean 10 kb), 15% error, Phred U[3,40]; scaled genome."""
    return dict(genome=max(30_000, int(5_000_000 * scale)), contigs=3, depth=(10, 200), mean=10_000, sd=4_000,
                err=0.15, qual_range=(3, 40))


def _workload(args):
    if args.config == 3:
        return {"workload": "window POA consensus, config 3 fragment correction (-f): %d bp genome in 3 contigs "
                            "(5 Mb x scale), depth 10-200x sinusoid, 15%% error FASTQ, all-vs-all dual PAF, "
                            "-w 500 -m 3 -x -5 -g -4" % _fragment_shape(args.scale)["genome"],
                "genome_scale": args.scale, "l2": "flushed between steps (512 MiB write); per-step scratch > L2"}
    return {"workload": "window POA consensus, config %d (%s)" % (args.config, {
        1: "1 Mb genome, 50x FASTQ 12% error, PAF +-50 bp, -w 500 -m 3 -x -5 -g -4",
        0: "50 kb genome, 30x FASTA 13% error, PAF, -w 500 -m 3 -x -5 -g -4"}[args.config]),
        "genome_scale": args.scale, "l2": "flushed between steps (512 MiB write); per-step scratch > L2"}


def _cpu_baseline(job_windows, n_sample, match, mismatch, gap):
    """The CPU oracle on the first n_sample windows with every host thread:
    (windows, seconds, DP cells, edge-cells, threads, [(consensus, polished)])."""
    import oracle
    blob = oracle.windows_blob(job_windows[:n_sample])
    threads = os.cpu_count() or 1
    n, sec, cells, ecells, res = oracle.consensus_blob_out(blob, n_sample, threads, match, mismatch, gap, True)
    return n, sec, cells, ecells, threads, res


def _serving_jobs(args):
    from racon_b200 import synthetic
    base = args.data_dir or os.path.join(tempfile.gettempdir(), "racon_b200_bench")
    d = os.path.join(base, "config4_n%d" % args.serving_jobs)
    marker = os.path.join(d, "done.json")
    if os.path.exists(marker):
        with open(marker) as fh:
            return json.load(fh)
    t0 = time.perf_counter()
    jobs = synthetic.serving_jobs(d, args.serving_jobs, seed=4)
    sys.stderr.write("[serving] generated %d jobs in %.1f s\n" % (len(jobs), time.perf_counter() - t0))
    with open(marker, "w") as fh:
        json.dump(jobs, fh)
    return jobs


def _pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return xs[k]


def run_serving(args, device, rates):
    """Config 4: a stream of config-0-like jobs through the serving loop.
    Isolated-job latency (each job alone on an idle server), peak throughput
    (all jobs at once), then Poisson arrivals at fractions of that peak; every
    output is checked against the job's isolated output."""
    import random
    import racon_b200
    jobs = _serving_jobs(args)
    w = 500
    windows = [(j[3]["draft_length"] + w - 1) // w for j in jobs]
    out = {"jobs": len(jobs), "workers": args.workers,
           "job_shape": "contig log-uniform 20 kb-2 Mb, coverage U[20,80], error U[8,15]%, FASTA, PAF, "
                        "-w 500 -m 3 -x -5 -g -4",
           "windows": sum(windows)}
    import torch
    free_b, _ = torch.cuda.mem_get_info(device)
    budget = int(free_b * 0.7)
    out["hbm_budget"] = budget
    out["shared_consensus"] = not args.no_shared_consensus
    out["shared_alignment"] = not args.no_shared_alignment
    out["alignment_ctas_per_sm"] = args.alignment_ctas or 1
    out["large_first_every"] = args.large_first_every
    out["alignment_yield"] = args.alignment_yield
    out["alignment_share"] = args.alignment_share
    t_start = time.perf_counter()

    def log(msg):
        sys.stderr.write("[serving %.1fs] %s\n" % (time.perf_counter() - t_start, msg))
        sys.stderr.flush()

    with racon_b200.Server(device, workers=args.workers, hbm_budget=budget, match=3, mismatch=-5, gap=-4,
                           window_length=w, shared_consensus=not args.no_shared_consensus,
                           alignment_yield=args.alignment_yield,
                           alignment_share=args.alignment_share,
                           shared_alignment=not args.no_shared_alignment,
                           alignment_ctas_per_sm=args.alignment_ctas,
                           large_first_every=args.large_first_every) as srv:
        def run(arrivals):
            t0 = time.perf_counter()
            tickets = []
            for i, j in enumerate(jobs):
                if arrivals is not None:
                    dt = arrivals[i] - (time.perf_counter() - t0)
                    if dt > 0:
                        time.sleep(dt)
                tickets.append(srv.submit(j[0], j[1], j[2]))
            res = [srv.wait(t) for t in tickets]
            span = max(r[1]["finished"] for r in res) - min(r[1]["submitted"] for r in res)
            return [r[0] for r in res], [r[1] for r in res], span

        log("server up, %d jobs, %d windows" % (len(jobs), sum(windows)))
        run(None)  # warm-up pass
        log("warm-up pass done")
        # every worker's buffers at the working size: the largest job once per
        # worker, all at once (an idle worker takes each)
        big = max(range(len(jobs)), key=lambda i: windows[i])
        for t in [srv.submit(*jobs[big][:3]) for _ in range(args.workers)]:
            srv.wait(t)
        log("workers warmed with the largest job")
        # each job alone, twice; the faster run is its isolated time
        iso, alone, iso_stage = [], [], []
        for j in jobs:
            best = None
            for _ in range(2):
                fasta, tm = srv.wait(srv.submit(j[0], j[1], j[2]))
                dt = tm["finished"] - tm["submitted"]
                if best is None or dt < best[0]:
                    best = (dt, fasta, list(tm["stage_seconds"]))
            iso.append(best[0])
            alone.append(best[1])
            iso_stage.append(best[2])
        log("isolated runs done, sum %.2f s" % sum(iso))
        fastas, _, span = run(None)
        assert fastas == alone, "a job's output differs between alone and in the mix"
        peak = len(jobs) / span
        log("peak run done, makespan %.2f s" % span)
        slow = max(range(len(jobs)), key=lambda k: iso[k])
        out.update(isolated_s={"p50": _pct(iso, 50), "max": max(iso), "sum": sum(iso),
                               "max_job": {"windows": windows[slow], "stage_s": iso_stage[slow]}},
                   peak={"jobs_per_s": peak, "windows_per_s": sum(windows) / span, "makespan_s": span})
        sweep = []
        rng = random.Random(4)
        for frac in rates:
            lam = frac * peak
            t, arrivals = 0.0, []
            for _ in jobs:
                arrivals.append(t)
                t += rng.expovariate(lam)
            fastas, times, span = run(arrivals)
            assert fastas == alone, "a job's output differs between alone and in the mix"
            lat = [tm["finished"] - tm["submitted"] for tm in times]
            ratio = [a / b for a, b in zip(lat, iso)]
            # where a job's time went: queueing for a worker, then the job's
            # stages on it (load, alignment + layers, window records, consensus)
            wait = [tm["admitted"] - tm["submitted"] for tm in times]
            stages = [[tm["stage_seconds"][k] for tm in times] for k in range(4)]
            log("load %.2f done, makespan %.2f s, p99 latency %.2f s" % (frac, span, _pct(lat, 99)))
            worst = max(range(len(jobs)), key=lambda k: ratio[k])
            sweep.append({"load": frac, "jobs_per_s": len(jobs) / span, "windows_per_s": sum(windows) / span,
                          "latency_s": {"p50": _pct(lat, 50), "p99": _pct(lat, 99)},
                          "latency_vs_isolated": {"p50": _pct(ratio, 50), "p99": _pct(ratio, 99)},
                          "admission_wait_s": {"mean": sum(wait) / len(wait), "max": max(wait)},
                          "stage_mean_s": [sum(x) / len(x) for x in stages],
                          "stage_max_s": [max(x) for x in stages],
                          "worst_job": {"windows": windows[worst], "isolated_s": iso[worst], "latency_s": lat[worst],
                                        "admission_wait_s": wait[worst],
                                        "stage_s": [stages[k][worst] for k in range(4)],
                                        "isolated_stage_s": list(iso_stage[worst])}})
        out["rates"] = sweep
    return out


def run_pipeline(args, paths, m, x, g, w):
    """The whole job end to end, as racon's wall time counts it (parse,
    overlap alignment, layers, consensus, stitching, FASTA text): the device
    path through rb_polish_files against the CPU oracle's pipeline on every
    host thread, and the two FASTA outputs compared byte for byte."""
    import racon_b200
    import oracle
    frag = args.config == 3
    kw = dict(window_length=w, quality_threshold=10.0, error_threshold=0.3, match=m, mismatch=x, gap=g)
    threads = os.cpu_count() or 1
    racon_b200.polish_files(*paths, fragment=frag, drop_unpolished=not frag, threads=threads, **kw)  # warm
    dev = []
    for _ in range(2):
        t0 = time.perf_counter()
        got = racon_b200.polish_files(*paths, fragment=frag, drop_unpolished=not frag, threads=threads, **kw)
        dev.append(time.perf_counter() - t0)
    t0 = time.perf_counter()
    want, stage_s, counts = oracle.polish(*paths, fragment=frag, drop_unpolished=not frag, threads=threads, **kw)
    cpu_s = time.perf_counter() - t0
    return {"device_s": min(dev), "oracle_s": cpu_s, "oracle_threads": threads, "speedup": cpu_s / min(dev),
            "fasta_identical": got == want, "fasta_bytes": len(got),
            "path": "rb_polish_files (parse -> device alignment -> device layers -> device consensus -> stitch) "
                    "vs the CPU oracle's pipeline, wall time per job"}


def _oracle_align(pairs, threads):
    """CPU oracle (edlib NW + path restatement) over pairs on `threads`
    threads (the ctypes call releases the GIL); returns seconds."""
    import concurrent.futures
    import oracle
    oracle.load()
    t0 = time.perf_counter()
    with concurrent.futures.ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda p: oracle.nw_cigar(p["query"], p["target"]), pairs))
    return time.perf_counter() - t0


def _align_workload(args):
    return {"workload": "overlap alignment batch, config 2 shape: %d pairs per step (the named batch is 100k), "
                        "target spans U[1 kb, 50 kb], query = span at 7%% sub + 4%% ins + 4%% del, edlib NW + "
                        "path, CIGAR + breakpoints every 500 bp" % args.pairs,
            "l2": "flushed between steps (512 MiB write); codes + scratch > L2"}


def run_align(args, local, world, rank):
    """Config 2: device overlap alignment (edit distance, CIGAR, breakpoints)."""
    import torch
    import racon_b200
    from racon_b200 import synthetic
    pairs = synthetic.pairs(args.pairs, 1_000, 50_000, seed=shard_seed(2, rank))
    nominal = sum(len(p["query"]) * len(p["target"]) for p in pairs)
    ctx = racon_b200.Context(local)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    ctx.align_stage(pairs, want_cigar=True)
    tuning = None if args.no_autotune else ctx.autotune(consensus=False, alignment=True)
    for _ in range(args.warmup):
        ctx.align_run()
    ref = ctx.align_fetch()
    clocks = Clocks(local)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks.start()
    kms, launches = [], 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ctx.align_run()
        st = ctx.align_stats()
        kms.append(st.kernel_ms)
        launches += st.launches
    torch.cuda.synchronize()
    clk = clocks.stop()
    assert ctx.align_fetch() == ref, "device results changed between steps"
    dev_s = sum(kms) / 1000.0
    t_max = max_over_ranks(dev_s, world)
    dev_s_max = t_max
    value = world * len(pairs) * args.steps / dev_s_max
    # end to end: rb_align_batch with host buffers (the rb_pair array over
    # the pairs' bytes is built once; each step is the C call: copy, H2D,
    # device encoding, kernels, D2H, results in host arrays)
    prepared = ctx.prepare_pairs(pairs)
    ctx.align_prepared(prepared, want_cigar=True)
    t0 = time.perf_counter()
    h2d = d2h = 0
    for _ in range(args.steps):
        r = ctx.align_prepared(prepared, want_cigar=True)
        st = ctx.align_stats()
        h2d += st.h2d_bytes
        d2h += st.d2h_bytes
    e2e_s = time.perf_counter() - t0
    assert ctx.aln_results(r, len(pairs), True) == ref
    # roofline: minimal Myers band of the final distance, ~34 int32 ops per
    # 64-row word and column
    words = 0
    for p, r in zip(pairs, ref):
        m, n, d = len(p["query"]), len(p["target"]), r["edit_distance"]
        words += n * -(-(2 * d + abs(m - n) + 1) // 64)
    peaks, _ = _peaks()
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    sm_mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    int_peak_tops = sm_count * 128 * sm_mhz * 1e6 / 1e12
    achieved_tops = words * 34 * args.steps / dev_s / 1e12
    in_bytes = sum(len(p["query"]) + len(p["target"]) for p in pairs)
    out_bytes = sum(len(r["cigar"]) + 8 * len(r["breakpoints"]) + 4 for r in ref)
    achieved_gbs = (in_bytes + out_bytes) * args.steps / dev_s / 1e9
    out = {"metric": "overlap alignment pairs/s", "value": value, "unit": "pairs/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dev_s_max / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 bit-vectors",
           "data": "synthetic (seeded)", "config": _align_workload(args),
           "gcups_nominal": nominal * args.steps / dev_s / 1e9, "gpu_launches": launches,
           "e2e": {"value": world * len(pairs) * args.steps / e2e_s, "unit": "pairs/s",
                   "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps},
           "roofline": {"bound": "hbm", "kernel": "nw_distance_kernel + nw_level_kernel",
                        "achieved": achieved_gbs, "peak": peaks.get("hbm_gbs", 6650.0), "unit": "GB/s",
                        "frac": achieved_gbs / peaks.get("hbm_gbs", 6650.0),
                        "traffic": nominal * NWD_DRAM_BYTES_PER_CELL,
                        "traffic_source": "nw_distance_kernel DRAM bytes per nominal cell from a 500-pair ncu "
                                          "capture, times this step's nominal cells",
                        "note": "algorithmic bytes = sequences in + CIGAR and breakpoints out; the sweep is "
                                "integer-issue bound, see compute"},
           "compute": {"bound": "int32 issue", "achieved_tops": achieved_tops, "peak_tops": int_peak_tops,
                       "frac": achieved_tops / int_peak_tops, "band_words": words,
                       "note": "minimal band of the final distance x 34 int32 ops per 64-row word"},
           "clocks": clk, "tuning": tuning}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample = pairs[:256]
        threads = os.cpu_count() or 1
        sec = _oracle_align(sample, threads)
        out["cpu_baseline"] = {"value": len(sample) / sec, "unit": "pairs/s", "cores": threads, "kind": "port",
                               "sample": "first %d of %d pairs, NW + path + CIGAR (CPU oracle)" % (len(sample),
                                                                                              len(pairs))}
    ctx.close()
    return out


def run_reference(args):
    world, rank, local = _dist()
    if rank != 0:
        return
    import oracle
    if args.config == 2:
        from racon_b200 import synthetic
        pairs = synthetic.pairs(min(args.pairs, 1024), 1_000, 50_000, seed=2)
        threads = os.cpu_count() or 1
        _oracle_align(pairs[:4], threads)
        secs = [_oracle_align(pairs, threads) for _ in range(args.steps)]
        value = len(pairs) * args.steps / sum(secs)
        print(json.dumps({"metric": "overlap alignment pairs/s", "value": value, "unit": "pairs/s",
                          "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": 1,
                          "ms_per_step": 1000 * sum(secs) / args.steps, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "u64 bit-vectors",
                          "data": "synthetic (seeded)", "config": _align_workload(args),
                          "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "port",
                                           "sample": "first %d pairs of the batch per step (CPU oracle)" % len(pairs)},
                          "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    if args.config == 4:
        # the CPU oracle polishes the config-4 jobs one after another (a bounded sample of the stream)
        jobs = _serving_jobs(args)
        threads = os.cpu_count() or 1
        done_w, total_s = 0, 0.0
        for j in jobs:
            t0 = time.perf_counter()
            oracle.polish(j[0], j[1], j[2], threads=threads)
            total_s += time.perf_counter() - t0
            done_w += (j[3]["draft_length"] + 499) // 500
            if total_s > 30:
                break
        value = done_w / total_s
        print(json.dumps({"metric": "serving windows/s at 80% load, p50/p99 job latency", "value": value,
                          "unit": "windows/s", "impl": "reference", "n_gpus": args.gpus, "steps": 1, "warmup": 0,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
                          "data": "synthetic (seeded)", "config": {"workload": "config 4 serving loop",
                                                                   "jobs": len(jobs)},
                          "cpu_baseline": {"value": value, "unit": "windows/s", "cores": threads, "kind": "port",
                                           "sample": "jobs polished back to back until 30 s (CPU oracle)"},
                          "e2e": {"value": value, "unit": "windows/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    paths = _data(args, 0)
    wins = oracle.dump_windows(*paths, fragment=args.config == 3, threads=os.cpu_count() or 1)
    n_sample = min(args.cpu_sample, len(wins))
    blob = oracle.windows_blob(wins[:n_sample])
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle.consensus_blob(blob, min(32, n_sample), threads, 3, -5, -4, True)
    total_n, total_s = 0, 0.0
    for _ in range(args.steps):
        n, sec, cells = oracle.consensus_blob(blob, n_sample, threads, 3, -5, -4, True)
        total_n += n
        total_s += sec
    value = total_n / total_s
    out = {"metric": "POA windows/s", "value": value, "unit": "windows/s", "impl": "reference",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1000 * total_s / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)", "config": _workload(args),
           "cpu_baseline": {"value": value, "unit": "windows/s", "cores": threads, "kind": "port",
                            "sample": "%d of %d windows per step (CPU oracle restatement; reference racon does not "
                                      "build here)" % (n_sample, len(wins))},
           "e2e": {"value": value, "unit": "windows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import racon_b200
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if args.config == 2:
        if world > 1:
            import datetime
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                                 device_id=torch.device("cuda", local))
        out = run_align(args, local, world, rank)
        if rank == 0:
            print(json.dumps(out))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.config == 4:
        # serving loop alone: load sweep over the config-4 job stream
        res = run_serving(args, local, [0.25, 0.5, 0.8, 1.0])
        best = max(r["windows_per_s"] for r in res["rates"])
        r80 = [r for r in res["rates"] if r["load"] == 0.8][0]
        if rank == 0:
            print(json.dumps({"metric": "serving windows/s at 80% load, p50/p99 job latency", "value": r80["windows_per_s"],
                              "unit": "windows/s", "n_gpus": world, "steps": 1, "warmup": 1,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
                              "data": "synthetic (seeded)", "config": {"workload": "config 4 serving loop",
                                                                       "jobs": res["jobs"]},
                              "p99_latency_vs_isolated": r80["latency_vs_isolated"]["p99"],
                              "best_windows_per_s": best, "serving": res}))
        return
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local))
    m, x, g, w = 3, -5, -4, 500
    paths = _data(args, rank)
    job = racon_b200.Job(*paths, fragment=args.config == 3, window_length=w, match=m, mismatch=x, gap=g,
                         device=local)
    n_win, n_layers, layer_bases, bb_bases = job.layer_stats()
    jst = job.device_stats()
    ctx = racon_b200.Context(local, m, x, g, w)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    # ---- device-resident throughput ----
    ctx.poa_stage_job(job)
    tuning = None
    if not args.no_autotune:
        # the device's launch choices measured on this job's windows (every
        # candidate gives the same consensus; checked inside rb_autotune)
        tuning = ctx.autotune(consensus=True)
    for _ in range(args.warmup):
        ctx.poa_run()
    reference_out = ctx.poa_fetch()
    clocks = Clocks(local)
    barrier()
    clocks.start()
    kms, launches, cells, ecells = [], 0, 0, 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ctx.poa_run()
        st = ctx.poa_stats()
        kms.append(st.kernel_ms)
        launches += st.launches
        cells += st.cells
        ecells += st.edge_cells
    barrier()
    clk = clocks.stop()
    assert ctx.poa_fetch() == reference_out, "device results changed between steps"
    dev_s = sum(kms) / 1000.0
    t_max = max_over_ranks(dev_s, world)
    dev_s_max = t_max
    value = world * n_win * args.steps / dev_s_max
    gcups = cells / dev_s / 1e9

    # ---- plain comparison form (one window per block, input order, no queue) ----
    ctx.poa_run(plain=True)
    plain_ms, plain_launches = [], 0
    barrier()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ctx.poa_run(plain=True)
        st = ctx.poa_stats()
        plain_ms.append(st.kernel_ms)
        plain_launches += st.launches
    barrier()
    assert ctx.poa_fetch() == reference_out, "plain form results differ from the batched form"
    t_max = max_over_ranks(sum(plain_ms) / 1000.0, world)
    plain_value = world * n_win * args.steps / t_max

    # ---- end to end through the C ABI with host buffers: the polishing
    # path (sequence table + breaking points in, layers assembled on the
    # device) ----
    def device_step():
        ctx.poa_stage_job_device(job)
        ctx.poa_run()
        res = ctx.poa_fetch()
        sq, ly, po = ctx.sequence_stats(), ctx.layer_stats(), ctx.poa_stats()
        return res, sq.h2d_bytes + ly.h2d_bytes + po.h2d_bytes, ly.d2h_bytes + po.d2h_bytes, ly

    device_step()
    barrier()
    t0 = time.perf_counter()
    h2d = d2h = 0
    layer_ms, layer_launches = [], 0
    for _ in range(args.steps):
        res, hb, db, ly = device_step()
        h2d += hb
        d2h += db
        layer_ms.append(ly.kernel_ms)
        layer_launches += ly.launches
    barrier()
    e2e_s = time.perf_counter() - t0
    t_max = max_over_ranks(e2e_s, world)
    e2e_value = world * n_win * args.steps / t_max
    assert res == reference_out, "device layer assembly changed the consensus"

    # ---- the same through rb_poa_batch with host-assembled windows ----
    ctx.poa_job(job)
    barrier()
    t0 = time.perf_counter()
    hh2d = hd2h = 0
    for _ in range(args.steps):
        res = ctx.poa_job(job)
        st = ctx.poa_stats()
        hh2d += st.h2d_bytes
        hd2h += st.d2h_bytes
    barrier()
    t_max = max_over_ranks(time.perf_counter() - t0, world)
    host_layers_value = world * n_win * args.steps / t_max
    assert res == reference_out

    # ---- roofline of the dominant kernel (poa_kernel) ----
    peaks, peak_kind = _peaks()
    cons_bytes = sum(len(c) for c, _ in reference_out)
    algo_bytes = bb_bases * 2 + layer_bases * 2 + cons_bytes  # bases + qualities in, consensus out
    launch_s = dev_s / max(1, launches)
    achieved_gbs = algo_bytes * (args.steps / max(1, launches)) / launch_s / 1e9
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    sm_mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    int_peak_tops = sm_count * 128 * sm_mhz * 1e6 / 1e12
    # counted work: edge-cells (|layer| x sum over the aligned rows of
    # 1 + predecessors, counted by the kernel) x 3 int32 ops (add, max,
    # compare-select per max-plus term)
    achieved_tops = ecells * 3 / dev_s / 1e12
    out = {
        "metric": "POA windows/s", "value": value, "unit": "windows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * dev_s_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
        "config": _workload(args),
        "gcups": gcups,
        "cells_per_step": cells // max(1, args.steps),
        "windows_per_step": n_win, "layers_per_step": n_layers,
        "gpu_launches": launches,
        "plain": {"value": plain_value, "unit": "windows/s", "ms_per_step": sum(plain_ms) / max(1, args.steps),
                  "launches_per_step": plain_launches // max(1, args.steps),
                  "form": "one window per one-warp block, input order, one launch per batch, no queue; "
                          "same per-window code, identical output (checked)"},
        "batched_vs_plain": value / plain_value,
        "e2e": {"value": e2e_value, "unit": "windows/s", "h2d_bytes_per_step": h2d // max(1, args.steps),
                "d2h_bytes_per_step": d2h // max(1, args.steps),
                "path": "rb_sequences_stage + rb_poa_stage_overlaps (device layer assembly) + rb_poa_run + "
                        "rb_poa_fetch"},
        "e2e_host_layers": {"value": host_layers_value, "unit": "windows/s",
                            "h2d_bytes_per_step": hh2d // max(1, args.steps),
                            "d2h_bytes_per_step": hd2h // max(1, args.steps),
                            "path": "rb_poa_batch with host-assembled windows"},
        "layer_assembly": {"kernel_ms_per_step": sum(layer_ms) / max(1, len(layer_ms)),
                           "launches_per_step": layer_launches // max(1, args.steps), "layers": n_layers},
        "roofline": {"bound": "hbm", "kernel": "poa_kernel", "achieved": achieved_gbs,
                     "peak": peaks.get("hbm_gbs", 6650.0), "unit": "GB/s",
                     "frac": achieved_gbs / peaks.get("hbm_gbs", 6650.0),
                     "traffic": cells / max(1, launches) * POA_DRAM_BYTES_PER_CELL,
                     "traffic_source": "ncu dram bytes of a 0.1-scale capture, scaled by DP cells per launch",
                     "peak_source": peak_kind,
                     "note": "algorithmic bytes = bases+qualities in + consensus out; the DP is integer-issue "
                             "bound, see compute"},
        "compute": {"bound": "int32 issue", "achieved_tops": achieved_tops, "peak_tops": int_peak_tops,
                    "frac": achieved_tops / int_peak_tops, "gcups": gcups,
                    "edge_cells_per_step": ecells // max(1, args.steps),
                    "edge_cells_per_cell": ecells / max(1, cells),
                    "issued_frac": cells * POA_THREAD_INST_PER_CELL / dev_s / 1e12 / int_peak_tops,
                    "issued_note": "executed thread instructions (per DP cell from an ncu capture) / device time, "
                                   "against the same issue peak",
                    "note": "achieved = edge-cells counted on the device (|layer| x sum_v (1 + in-degree v) over "
                            "the aligned graph) x 3 int32 ops / device time; peak = SMs x 128 int32 lanes x median "
                            "SM clock under load"},
        "clocks": clk,
        "tuning": tuning,
        "stages_s": {"load": job.stage_seconds[0], "align": job.stage_seconds[1], "layers": job.stage_seconds[2],
                     "note": "align = sequence table to the device, overlap alignment and (PAF/MHAP) the "
                             "device layer assembly; layers = the host's window records"},
        "job_device_ms": {"align_kernels": jst["align"].kernel_ms, "align_h2d": jst["align"].h2d_ms,
                          "align_d2h": jst["align"].d2h_ms, "align_launches": jst["align"].launches,
                          "sequences_h2d": jst["sequences"].h2d_ms, "layer_kernels": jst["layers"].kernel_ms},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample = [job.window(i) for i in range(min(args.cpu_sample, n_win))]
        n, sec, ccells, cpu_ecells, threads, cpu_res = _cpu_baseline(sample, len(sample), m, x, g)
        out["cpu_baseline"] = {"value": n / sec, "unit": "windows/s", "cores": threads, "kind": "port",
                               "gcups": ccells / sec / 1e9,
                               "sample": "first %d of %d windows, one pass (CPU oracle restatement of racon's "
                                         "algorithm; reference racon does not build here)" % (n, n_win)}
        # parity on the timed workload: the oracle's consensus of the sampled
        # windows against the device's from the timed steps
        mism = sum(1 for a, b in zip(cpu_res, reference_out[:n]) if a != b)
        out["parity"] = {"windows_checked": n, "mismatches": mism,
                         "against": "CPU oracle, window by window (consensus bytes and polished flag)"}
        # the same work unit counted by the oracle on its sample, beside the
        # device's count over the whole step
        out["compute"]["oracle_sample_edge_cells_per_cell"] = cpu_ecells / max(1, ccells)
    ctx.close()
    job.close()
    if rank == 0 and world == 1 and not args.no_pipeline:
        out["pipeline"] = run_pipeline(args, paths, m, x, g, w)
    if world == 1 and args.serving_jobs > 0:
        # config 4 serving loop at 80% of its measured peak (--config 4 sweeps the load)
        out["serving"] = run_serving(args, local, [0.8])
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
