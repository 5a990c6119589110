#!/usr/bin/env python
"""Benchmark of the batched ML-KEM NTT + iNTT engine (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): 262,144
polynomials per GPU (N=256 int16 coefficients, seeded uniform in [0, q)),
forward NTT and inverse NTT as separate batched launches.  A step is one
forward launch plus one inverse launch over 262,144 polynomials each; the
value is round trips per second (polys/s), summed over ranks (weak scaling:
every rank owns its own 262,144-polynomial batches, there is no exchange).

L2 hygiene: four resident batches (4 x 128 MiB) rotate, so every launch reads
a batch last touched three launches earlier (384 MiB of traffic in between,
above the 126 MB L2).

Timing: --repeats regions of exactly --steps steps each, every region
bracketed by a barrier and a synchronize; the value is the median region (max
over ranks), with min and max beside it.  --gpus N without a launcher starts N
ranks itself through torch.distributed.run (one per GPU); under a launcher
--gpus must equal the number of ranks.

Beside the value (rank 0, one GPU): the reference's C on the host cores (all
threads and one thread) and the reference's own GPU kernels on the same GPU
(oracle/_ref/ntt_bench, built for sm_100a from ntt_bench/ntt_bench.cu).

--impl reference times the reference's own C ntt()/invntt()
(ntt_bench/ref, compiled unmodified into oracle/_ref) on all host threads, a
4096-polynomial sample of the same workload per step, in one process on rank
0's host whatever --gpus is.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

Q = 3329
METRIC = "NTT+iNTT polys/s & %HBM roofline (bit-exact), 1xB200; batched p50/p99 us"
BYTES_PER_POLY = 1024          # one transform: 512 B read + 512 B write
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20000)
    p.add_argument("--warmup", type=int, default=200)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--npoly", type=int, default=262144)
    p.add_argument("--repeats", type=int, default=7,
                   help="timed regions of --steps steps each; value = the median region")
    p.add_argument("--e2e-steps", type=int, default=30)
    p.add_argument("--no-reference-gpu", action="store_true",
                   help="skip the reference's own GPU kernels (oracle/_ref/ntt_bench)")
    p.add_argument("--cpu-seconds", type=float, default=6.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--variant", type=int, default=-1,
                   help="force a kernel variant in both directions (-1: auto; 0-3 mma.sync "
                        "shapes, 4 tcgen05)")
    p.add_argument("--fwd-variant", type=int, default=-1, help="force the forward's variant")
    p.add_argument("--inv-variant", type=int, default=-1, help="force the inverse's variant")
    p.add_argument("--sweep", action="store_true",
                   help="batch-size sweep 2^0..2^sweep-max (autotuned), JSON lines to --sweep-out")
    p.add_argument("--sweep-max", type=int, default=24)
    p.add_argument("--sweep-out", default="sweep.jsonl")
    p.add_argument("--matvec", action="store_true",
                   help="fused ML-KEM matrix-vector jobs, k ~ U{2,3,4} (eager and CUDA graph)")
    p.add_argument("--jobs", type=int, default=65536)
    p.add_argument("--chunk", type=int, default=0, help="tk_matvec chunk (vector polys), 0 = default")
    p.add_argument("--matvec-mode", type=int, default=2,
                   help="0 pipeline, 1 fused single launch, 2 tiled (the default)")
    p.add_argument("--forms", action="store_true",
                   help="forward NTT by input form (int16, small, packed 2/3-bit)")
    p.add_argument("--serve", action="store_true",
                   help="serving loop: Poisson arrivals at swept rates, server vs plain per-request")
    p.add_argument("--serve-requests", type=int, default=3000, help="requests per rate point")
    p.add_argument("--serve-rates", default="0.25,0.5,0.9,1.5,3,6",
                   help="offered load as multiples of the plain per-request capacity")
    p.add_argument("--serve-templates", type=int, default=256)
    p.add_argument("--serve-zero-copy", action="store_true")
    p.add_argument("--serve-no-arena", action="store_true",
                   help="skip the server arm whose requests lie back to back in one pinned arena")
    p.add_argument("--serve-plain-mode", type=int, default=2,
                   help="matrix-vector mode of the plain per-request path (0, 1, 2 as --matvec-mode)")
    p.add_argument("--traffic", action="store_true",
                   help="each direction's launch followed by a read-only pass over 4x the L2, "
                        "--steps times (for ncu --cache-control none: the pass's DRAM writes "
                        "are the launch's write-back)")
    return p.parse_args()


def config(npoly, world):
    return {
        "workload": f"batched forward NTT + inverse NTT as separate launches, {npoly} "
                    "polynomials per GPU (N=256 int16, uniform [0,q), q=3329)",
        "npoly_per_gpu": npoly,
        "global_batch": npoly * world,
        "parallelism": f"replicas/range-sharded x{world} (no collective on the data path)",
        "l2": "4 resident batches rotated per launch (512 MiB working set > 126 MB L2)",
    }


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """SM clock, power and clock-event reasons of one GPU while it runs: NVML
    polled every 2 ms from a thread (so that even a timed region of a few
    milliseconds gets samples), or nvidia-smi at 100 ms where NVML cannot be
    loaded.  The GPU is found by its PCI bus id, so the CUDA device number
    need not be NVML's index.  Reads only; changes no setting."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.device)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.stop_flag = threading.Event()

            def one():
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx,
                                  [n for n, bit in zip(self.REASONS, bits) if r & bit]))

            def poll():
                while not self.stop_flag.is_set():
                    one()
                    time.sleep(0.002)
            self.sample_now = one
            # the poller must get the interpreter while the caller launches
            self.switch = sys.getswitchinterval()
            sys.setswitchinterval(0.001)
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        fd, self.path = tempfile.mkstemp(prefix="tk_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.4)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.sample_now()  # at least one sample at the end of the window
            self.stop_flag.set()
            self.thread.join(timeout=10)
            sys.setswitchinterval(self.switch)
            if not self.rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                        "source": "nvml"}
            return {"sm_mhz": statistics.median(r[0] for r in self.rows),
                    "sm_max_mhz": max(r[1] for r in self.rows),
                    "reasons": sorted({n for r in self.rows for n in r[2]}),
                    "samples": len(self.rows), "source": "nvml, every 2 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = sorted({self.REASONS[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi, every 100 ms"}


def load_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def load_traffic(kernel: str, npoly: int):
    """DRAM bytes per launch from the committed ncu summary (per polynomial,
    scaled to this launch)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            per_poly = json.load(f)[kernel]["dram_bytes_per_poly"]
        return per_poly * npoly
    except Exception:
        return None


# ------------------------------------------------------------- CPU sides ----
def cpu_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import py_oracle
    o = py_oracle.Oracle()
    if py_oracle.RefKyber.available():
        r = py_oracle.RefKyber(3)
        return o, r.fn("ntt"), r.fn("invntt"), "reference"
    return o, o.fn("tko_ntt"), o.fn("tko_invntt"), "port"


def sample_input(n, seed=20240816):
    import numpy as np
    return np.random.default_rng(seed).integers(0, Q, size=(n, 256), dtype=np.int16)


def cpu_baseline(seconds: float):
    """The reference's C ntt() then invntt() on the host cores: all threads,
    and one thread (its per-core rate)."""
    o, f, i, kind = cpu_oracle()
    threads = os.cpu_count() or 1
    sample = sample_input(4096)
    rate, done = o.time_roundtrip(f, i, sample, threads, seconds)
    one = max(1.0, seconds / 2)
    rate1, done1 = o.time_roundtrip(f, i, sample, 1, one)
    return {"value": rate, "unit": "polys/s", "cores": threads, "kind": kind,
            "sample": f"NTT+iNTT round trips over a 4096-polynomial sample per thread, "
                      f"repeated for {seconds:.0f} s on {threads} threads ({done} polys)",
            "one_core": {"value": rate1, "unit": "polys/s", "cores": 1,
                         "sample": f"the same on one thread for {one:.0f} s ({done1} polys)"}}


def reference_gpu(npoly: int, runs: int = 30):
    """The reference's own GPU benchmark (ntt_bench/ntt_bench.cu:909-991, its
    kernels built unmodified for sm_100a into oracle/_ref/ntt_bench), run on
    this GPU at the same batch size; its summary table is parsed (median
    polys/s of NTT, iNTT and the round trip, per variant; the reference times
    every launch with its own events, ntt_bench/ntt_bench.cu:637-661)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ntt_bench")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ntt_bench not built (make -C oracle gpubar)"}
    try:
        p = subprocess.run([exe, str(npoly), str(runs)], capture_output=True, text=True,
                           timeout=300)
    except subprocess.TimeoutExpired:
        return {"unavailable": "ntt_bench did not finish in 300 s"}
    rows = {}
    in_table = False
    for line in p.stdout.splitlines():
        if line.startswith(" SUMMARY"):
            in_table = True
            continue
        if not in_table or "|" not in line or line.startswith("Variant") or line.startswith("-"):
            continue
        parts = [x.strip() for x in line.split("|")]
        try:
            nums = [float(v) for v in parts[1].split() + parts[2].split() + parts[3].split()]
        except (ValueError, IndexError):
            continue
        name = parts[0][:30].strip()   # %-30s variant label, then geometry and block
        ok = parts[4].split() if len(parts) > 4 else []
        rows[name] = {"ntt_med_polys_s": nums[1] * 1e6, "intt_med_polys_s": nums[3] * 1e6,
                      "roundtrip_med_polys_s": nums[5] * 1e6,
                      "parity_ok": ok == ["ok", "ok"]}
    if p.returncode != 0 or not rows:
        return {"unavailable": f"ntt_bench exited {p.returncode} ({len(rows)} rows parsed)",
                "stdout_tail": p.stdout[-400:]}
    best = max(rows, key=lambda k: rows[k]["roundtrip_med_polys_s"])
    return {"value": rows[best]["roundtrip_med_polys_s"], "unit": "polys/s",
            "best_variant": best, "npoly": npoly, "runs": runs, "variants": rows,
            "how": "oracle/_ref/ntt_bench <npoly> <runs>: the reference's kernels built for "
                   "sm_100a, run on this GPU; median round trip of its best variant"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    o, f, i, kind = cpu_oracle()
    threads = os.cpu_count() or 1
    sample = sample_input(4096)
    for _ in range(args.warmup):
        o.split_roundtrip(f, i, sample, threads)
    times = [o.split_roundtrip(f, i, sample, threads) for _ in range(args.steps)]
    total = sum(times)
    value = 4096 * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "polys/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "int16", "data": "synthetic",
        "config": config(args.npoly, world),
        "cpu_processes": 1,
        "note": "one CPU process on rank 0's host at every --gpus: the reference's C "
                "ntt()/invntt() has no GPU path, so its value does not grow with N",
        "cpu_baseline": {"value": value, "unit": "polys/s", "cores": threads, "kind": kind,
                         "sample": "each step: NTT then iNTT on a 4096-polynomial sample "
                                   f"of the workload, split over {threads} threads"},
        "e2e": {"value": value, "unit": "polys/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "latency_us": {"p50": 1e6 * statistics.median(times),
                       "p99": 1e6 * sorted(times)[min(len(times) - 1, int(0.99 * len(times)))]},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- ours ---
def apply_variants(tk, args):
    fwd = args.fwd_variant if args.fwd_variant >= 0 else args.variant
    inv = args.inv_variant if args.inv_variant >= 0 else args.variant
    if fwd >= 0:
        tk.set_variant(tk.FORWARD, fwd)
    if inv >= 0:
        tk.set_variant(tk.INVERSE, inv)


def run_ours(args):
    import numpy as np
    import torch

    import tensorkyber_b200 as tk

    from tensorkyber_b200 import dist as tkdist

    rank, world, local = tkdist.env()
    torch.cuda.set_device(local)
    # one process per GPU; NCCL only carries the barrier and the timing max
    dist = tkdist.init("nccl", 120.0, device=torch.device("cuda", local))
    tk.init(local)
    apply_variants(tk, args)
    n = args.npoly
    gen = np.random.default_rng(1000 + rank)
    batches = [torch.from_numpy(gen.integers(0, Q, size=(n, 256), dtype=np.int16)).cuda()
               for _ in range(4)]
    stream = torch.cuda.current_stream()

    def step(k):
        tk.ntt(batches[(2 * k) % 4], stream=stream)
        tk.invntt(batches[(2 * k + 1) % 4], stream=stream)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()

    K = args.steps
    R = max(1, args.repeats)
    # timed regions: R regions of exactly K steps back to back (no events
    # between the launches, so consecutive kernels overlap prologue and tail
    # through programmatic launch), each bracketed by a barrier and a
    # synchronize; the value is the median region (max over ranks per region)
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    sampler.start()
    region_ms = []
    for _ in range(R):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e_start.record(stream)
        for k in range(K):
            step(k)
        e_end.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        region_ms.append(e_start.elapsed_time(e_end))
    clocks = sampler.stop()
    # per-launch split (batch latency p50/p99): the same workload with an event
    # around each launch, which serialises the launches
    K2 = min(K, 2000)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * K2 + 1)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    for k in range(K2):
        tk.ntt(batches[(2 * k) % 4], stream=stream)
        ev[2 * k + 1].record(stream)
        tk.invntt(batches[(2 * k + 1) % 4], stream=stream)
        ev[2 * k + 2].record(stream)
    torch.cuda.synchronize()
    fwd_ms = [ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(K2)]
    inv_ms = [ev[2 * k + 1].elapsed_time(ev[2 * k + 2]) for k in range(K2)]
    # per-kernel average launch duration (roofline): K2 launches of one kernel
    # back to back between two events, batches rotated as in the timed region
    # (each launch reads data last touched three launches earlier, > L2)
    group_ms = {}
    for name, fn in (("ntt_fwd", tk.ntt), ("ntt_inv", tk.invntt)):
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        g0.record(stream)
        for k in range(K2):
            fn(batches[k % 4], stream=stream)
        g1.record(stream)
        torch.cuda.synchronize()
        group_ms[name] = g0.elapsed_time(g1) / K2
    region_ms = [tkdist.max_over_ranks(t, dist, device="cuda") for t in region_ms]
    total_ms = statistics.median(region_ms)
    status = tk.device_status(local)
    if status:
        raise RuntimeError(f"kernel status flags {status:#x}")

    # end to end through the host-memory API: pinned host batch in, result out
    e2e = None
    if args.e2e_steps > 0:
        host = torch.from_numpy(gen.integers(0, Q, size=(n, 256), dtype=np.int16)).pin_memory()
        h = host.numpy()
        tk.ntt_host(h)
        tk.invntt_host(h)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            tk.ntt_host(h)
            tk.invntt_host(h)
        e2e_s = tkdist.max_over_ranks(time.perf_counter() - t0, dist, device="cuda")
        e2e = {"value": world * n * args.e2e_steps / e2e_s, "unit": "polys/s",
               "h2d_bytes_per_step": 2 * n * 512, "d2h_bytes_per_step": 2 * n * 512,
               "steps": args.e2e_steps,
               "how": "tk_ntt_host + tk_invntt_host on a pinned host batch, wall clock"}

    if rank == 0:
        fwd_iso = sum(fwd_ms) / K2
        inv_iso = sum(inv_ms) / K2
        fwd_avg, inv_avg = group_ms["ntt_fwd"], group_ms["ntt_inv"]
        dom, avg = ("ntt_fwd", fwd_avg) if fwd_avg >= inv_avg else ("ntt_inv", inv_avg)
        peak, peak_kind = load_peak()
        achieved = BYTES_PER_POLY * n / (avg * 1e-3) / 1e9
        traffic = load_traffic(dom, n)
        lat_rt = sorted(f + i for f, i in zip(fwd_ms, inv_ms))
        line = {
            "metric": METRIC,
            "value": world * n * K / (total_ms * 1e-3),
            "unit": "polys/s",
            "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": total_ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int16", "data": "synthetic",
            "config": config(n, world),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6650 GB/s",
                         "bytes_per_launch": BYTES_PER_POLY * n,
                         "traffic_how": "ncu --cache-control none on this kernel at 262144 "
                                        "polynomials (bench.py --traffic): the launch's DRAM "
                                        "read + write plus the write-back drained after it, "
                                        "per polynomial, times this launch's polynomials"},
            "kernels_ms": {"ntt_fwd_avg": fwd_avg, "ntt_inv_avg": inv_avg,
                           "ntt_fwd_isolated": fwd_iso, "ntt_inv_isolated": inv_iso,
                           "how": "avg: K2 launches of one kernel back to back between two "
                                  "events; isolated: an event around every launch"},
            "kernel_variant": {"forward": tk.variant_name(tk.get_variant(tk.FORWARD, n)),
                               "inverse": tk.variant_name(tk.get_variant(tk.INVERSE, n))},
            "latency_us": {"batch_roundtrip_p50": 1e3 * lat_rt[len(lat_rt) // 2],
                           "batch_roundtrip_p99": 1e3 * lat_rt[min(K2 - 1, int(0.99 * K2))]},
            "e2e": e2e,
            "gpu_launches": 2 * K,
            "repeats": {"regions": R, "steps_per_region": K,
                        "ms_per_step_min": min(region_ms) / K,
                        "ms_per_step_median": total_ms / K,
                        "ms_per_step_max": max(region_ms) / K,
                        "how": "value and ms_per_step from the median of R timed regions of "
                               "K steps each (gpu_launches counts one region)"},
            "kernel_split_steps": K2,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
        if world == 1 and not args.no_reference_gpu:
            torch.cuda.synchronize()
            line["reference_gpu"] = reference_gpu(n)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_sweep(args):
    """Batch-size sweep: for every power of two up to 2^sweep-max, forward,
    inverse and round-trip throughput with the autotuned variant, and every
    variant's time per launch in each direction (mma.sync 0-3, tcgen05 4), as
    JSON lines (one per size) in --sweep-out; the summary line goes to stdout."""
    import torch

    import tensorkyber_b200 as tk

    torch.cuda.set_device(0)
    tk.init(0)
    t0 = time.perf_counter()
    tk.autotune(max_npoly=1 << min(args.sweep_max, 22), device=0)
    tune_s = time.perf_counter() - t0
    peak, peak_kind = load_peak()
    stream = torch.cuda.current_stream()
    rows = []
    with open(args.sweep_out, "w") as out:
        for b in range(args.sweep_max + 1):
            n = 1 << b
            nb = 4 if 4 * n * 512 <= (40 << 30) else 2
            batches = [torch.randint(0, Q, (n, 256), dtype=torch.int16, device="cuda")
                       for _ in range(nb)]
            # ~0.2 s of work per measurement, at least 20 launches
            K = max(20, min(4000, int(0.1 / max(n * 1024 / (peak * 1e9 * 0.7), 6e-6))))
            res = {}
            for name, fns in (("fwd", (tk.ntt,)), ("inv", (tk.invntt,)),
                              ("roundtrip", (tk.ntt, tk.invntt))):
                for k in range(3):
                    for f in fns:
                        f(batches[k % nb], stream=stream)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                for k in range(K):
                    for j, f in enumerate(fns):
                        f(batches[(len(fns) * k + j) % nb], stream=stream)
                e1.record(stream)
                torch.cuda.synchronize()
                res[name] = e0.elapsed_time(e1) * 1e3 / K   # us per step
            # every variant in each direction at this size (the autotuner's
            # candidates: mma.sync shapes 0-3, tcgen05 4), K launches each
            per_variant = {}
            for dname, d, f in (("fwd", tk.FORWARD, tk.ntt), ("inv", tk.INVERSE, tk.invntt)):
                per_variant[dname] = {}
                for v in range(tk.variant_count()):
                    tk.set_variant(d, v)
                    for k in range(3):
                        f(batches[k % nb], stream=stream)
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    for k in range(K):
                        f(batches[k % nb], stream=stream)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    per_variant[dname][str(v)] = e0.elapsed_time(e1) * 1e3 / K
                tk.set_variant(d, -1)
            row = {
                "npoly": n,
                "fwd_us": res["fwd"], "inv_us": res["inv"], "roundtrip_us": res["roundtrip"],
                "variant_us": per_variant,
                "polys_per_s": n / (res["roundtrip"] * 1e-6),
                "hbm_frac": (2 * n * 1024 / (res["roundtrip"] * 1e-6)) / (peak * 1e9),
                "l2_resident": nb * n * 512 < (126 << 20),
                "variant": {"fwd": tk.get_variant(tk.FORWARD, n),
                            "inv": tk.get_variant(tk.INVERSE, n)},
                "steps": K,
            }
            rows.append(row)
            out.write(json.dumps(row) + "\n")
            out.flush()
            del batches
            torch.cuda.empty_cache()
    big = [r for r in rows if r["npoly"] >= (1 << 20)]
    print(json.dumps({
        "metric": "batch-size sweep NTT+iNTT polys/s and %HBM roofline (autotuned variants)",
        "points": len(rows), "out": args.sweep_out, "autotune_s": tune_s,
        "peak_gbs": peak, "peak_source": peak_kind,
        "best_polys_per_s": max(r["polys_per_s"] for r in rows),
        "min_hbm_frac_at_2^20_plus": min(r["hbm_frac"] for r in big) if big else None,
    }), flush=True)


def run_traffic(args):
    """DRAM traffic of one launch including its write-back.  The L2 is
    write-back: part of a launch's output is still dirty in L2 when the launch
    ends and reaches DRAM later, inside whichever kernel evicts it.  Here every
    launch is followed by a read-only pass (a sum) over a buffer four times the
    L2, which evicts every dirty line and writes nothing of its own, so under
    `ncu --cache-control none` a launch's whole traffic is its own
    dram__bytes_read.sum + dram__bytes_write.sum plus the pass's
    dram__bytes_write.sum.  Prints the configuration; the figures come from
    ncu."""
    import numpy as np
    import torch

    import tensorkyber_b200 as tk

    torch.cuda.set_device(0)
    tk.init(0)
    apply_variants(tk, args)
    n = args.npoly
    gen = np.random.default_rng(1000)
    data = torch.from_numpy(gen.integers(0, Q, size=(n, 256), dtype=np.int16)).cuda()
    drain = torch.ones(4 * 126 * 2**20 // 4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    total = torch.zeros((), dtype=torch.int64, device="cuda")
    drain.sum()                      # the drain buffer itself clean before the first launch
    torch.cuda.synchronize()
    for _ in range(args.steps):
        tk.ntt(data, stream=stream)
        total += drain.sum()
        tk.invntt(data, stream=stream)
        total += drain.sum()
    torch.cuda.synchronize()
    status = tk.device_status(0)
    if status:
        raise RuntimeError(f"kernel status flags {status:#x}")
    print(json.dumps({
        "metric": "DRAM traffic per launch incl. write-back (read with ncu)",
        "npoly": n, "steps": args.steps, "drain_bytes": drain.numel() * 4,
        "kernel_variant": {"forward": tk.variant_name(tk.get_variant(tk.FORWARD, n)),
                           "inverse": tk.variant_name(tk.get_variant(tk.INVERSE, n))},
        "sequence": "ntt, sum(drain), invntt, sum(drain) per step",
    }), flush=True)


def run_forms(args):
    """Forward NTT by input form at --npoly polynomials (default 2^20): int16
    (tk_ntt), small int16 in [-128, 127] (tk_ntt_small, single-limb stage 1),
    packed 2-bit and 3-bit fields (tk_ntt_packed).  Inputs are seeded ternary
    ([-1, 1]) polynomials, the same ones in every form; four rotating input and
    output batches (above L2).  Algorithmic bytes per polynomial: input row
    (512 / 64 / 128) + 512 output.  Outputs are checked equal across forms."""
    import numpy as np
    import torch

    import tensorkyber_b200 as tk

    torch.cuda.set_device(0)
    tk.init(0)
    n = args.npoly if args.npoly != 262144 else 1 << 20
    peak, peak_kind = load_peak()
    stream = torch.cuda.current_stream()
    x = np.random.default_rng(2026).integers(-1, 2, size=(n, 256)).astype(np.int16)
    nb = 4
    srcs = {"int16": [torch.from_numpy(x).cuda() for _ in range(nb)],
            "small": None,
            "pack2": [torch.from_numpy(tk.pack_small(x, 2)).cuda() for _ in range(nb)],
            "pack3": [torch.from_numpy(tk.pack_small(x, 3)).cuda() for _ in range(nb)]}
    srcs["small"] = srcs["int16"]
    outs = [torch.empty((n, 256), dtype=torch.int16, device="cuda") for _ in range(nb)]
    in_bytes = {"int16": 512, "small": 512, "pack2": 64, "pack3": 128}
    call = {"int16": lambda s, o: tk.ntt(s, out=o, stream=stream),
            "small": lambda s, o: tk.ntt_small(s, o, stream=stream),
            "pack2": lambda s, o: tk.ntt_packed(s, 2, o, stream=stream),
            "pack3": lambda s, o: tk.ntt_packed(s, 3, o, stream=stream)}
    K = args.steps if args.steps != 20000 else 400
    res, ref = {}, None
    sampler = ClockSampler(0)
    sampler.start()
    for name in ("int16", "small", "pack2", "pack3"):
        for k in range(max(3, args.warmup if args.warmup != 200 else 5)):
            call[name](srcs[name][k % nb], outs[k % nb])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(K):
            call[name](srcs[name][k % nb], outs[k % nb])
        e1.record(stream)
        torch.cuda.synchronize()
        us = e0.elapsed_time(e1) * 1e3 / K
        got = outs[(K - 1) % nb].cpu().numpy()
        if ref is None:
            ref = got
        assert (got == ref).all(), name
        gbs = n * (in_bytes[name] + 512) / (us * 1e-6) / 1e9
        res[name] = {"us_per_launch": us, "polys_per_s": n / (us * 1e-6),
                     "bytes_per_poly": in_bytes[name] + 512, "achieved_gbs": gbs,
                     "hbm_frac": gbs / peak}
    clocks = sampler.stop()
    assert tk.device_status(0) == 0
    print(json.dumps({
        "metric": "forward NTT polys/s by input form, 1xB200", "npoly": n, "steps": K,
        "forms": res, "outputs_equal_across_forms": True, "peak_gbs": peak,
        "peak_source": peak_kind, "clocks": clocks, "dtype": "int16", "data": "synthetic",
        "config": {"workload": f"{n} ternary polynomials, 4 rotating batches (> L2)"},
    }), flush=True)


def run_matvec(args):
    """Mixed-k ML-KEM matrix-vector jobs: out_i = invntt(sum_j A_ij o ntt(s_j)) + e_i,
    k drawn uniformly from {2, 3, 4} (seeded), A uniform in [0, q), s and e in
    [-3, 3]; one tk_matvec call (three uniform-k batches) per step, timed eagerly
    and as a replayed CUDA graph."""
    import numpy as np
    import torch

    import tensorkyber_b200 as tk

    torch.cuda.set_device(0)
    tk.init(0)
    tk.set_option(tk.OPT_MATVEC_CHUNK_POLYS, args.chunk)
    tk.set_option(tk.OPT_MATVEC_MODE, args.matvec_mode)
    ks = np.random.default_rng(2024).integers(2, 5, size=args.jobs)
    g = torch.Generator(device="cuda").manual_seed(7)
    batches, nbytes = [], 0
    for k in (2, 3, 4):
        n = int((ks == k).sum())
        A = torch.randint(0, Q, (n, k, k, 256), dtype=torch.int16, device="cuda", generator=g)
        sv = torch.randint(-3, 4, (n, k, 256), dtype=torch.int16, device="cuda", generator=g)
        e = torch.randint(-3, 4, (n, k, 256), dtype=torch.int16, device="cuda", generator=g)
        out = torch.empty_like(sv)
        batches.append((k, A, sv, e, out))
        nbytes += n * (k * k + 3 * k) * 512
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        tk.matvec(batches, stream=stream)
    torch.cuda.synchronize()
    K = args.steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(0)
    sampler.start()
    e0.record(stream)
    for _ in range(K):
        tk.matvec(batches, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    eager_ms = e0.elapsed_time(e1) / K
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        tk.matvec(batches, stream=side)          # warm the side stream
    torch.cuda.synchronize()
    with torch.cuda.graph(graph):
        tk.matvec(batches)
    graph.replay()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(K):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    graph_ms = e0.elapsed_time(e1) / K
    clocks = sampler.stop()
    peak, peak_kind = load_peak()
    assert tk.device_status(0) == 0
    achieved = nbytes / (graph_ms * 1e-3) / 1e9
    print(json.dumps({
        "metric": "fused ML-KEM matrix-vector jobs/s (k ~ U{2,3,4}), 1xB200",
        "value": args.jobs / (graph_ms * 1e-3), "unit": "jobs/s", "n_gpus": 1,
        "steps": K, "warmup": args.warmup, "ms_per_step": graph_ms, "higher_is_better": True,
        "eager_ms_per_step": eager_ms, "eager_jobs_per_s": args.jobs / (eager_ms * 1e-3),
        "jobs_per_k": {str(k): int((ks == k).sum()) for k in (2, 3, 4)},
        "config": {"workload": f"{args.jobs} jobs, A k x k uniform [0,q) NTT domain, s,e in [-3,3]",
                   "chunk_vec_polys": tk.get_option(tk.OPT_MATVEC_CHUNK_POLYS),
                   "mode": ["pipeline", "fused", "tiled"][tk.get_option(tk.OPT_MATVEC_MODE)]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "bytes_per_step": nbytes,
                     "peak_source": peak_kind},
        "clocks": clocks, "dtype": "int16", "data": "synthetic",
    }), flush=True)


def run_serve(args):
    """Serving loop against the plain per-request launch, on the same requests.

    A request is njobs ~ U{1..64} matrix-vector jobs of one k ~ U{2,3,4} with
    every coefficient uniform in [0, q) (seeded), in pinned host memory, its
    A, s and e back to back in one buffer (one copy in, for both arms).
    Arrivals are Poisson at a rate swept as multiples of the plain path's
    measured capacity.  Plain: one host thread serves requests in arrival
    order, each as tk_matvec_host (copy in, one fused launch, copy out, sync).
    Server: the same thread submits each request at its arrival time to
    tk_server (continuous batching; staged through the server's HBM pool, and
    with --serve-zero-copy also a server that reads the pinned buffers in
    place).  Latency = completion - scheduled
    arrival; throughput = output polynomials / (last completion - start)."""
    import ctypes

    import numpy as np
    import torch

    import tensorkyber_b200 as tk

    torch.cuda.set_device(0)
    tk.init(0)
    tk.set_option(tk.OPT_MATVEC_MODE, args.serve_plain_mode)
    L = tk.lib()
    r = np.random.default_rng(2025)
    T = args.serve_templates

    def pinned(shape):
        return torch.empty(shape, dtype=torch.int16, pin_memory=True).numpy()

    tmpl = []
    for _ in range(T):
        k, n = int(r.integers(2, 5)), int(r.integers(1, 65))
        blk = pinned((n * (k * k + 2 * k), 256))       # one request message: A | s | e
        A = blk[:n * k * k].reshape(n, k, k, 256)
        sv = blk[n * k * k:n * (k * k + k)].reshape(n, k, 256)
        e = blk[n * (k * k + k):].reshape(n, k, 256)
        A[...] = r.integers(0, Q, size=A.shape)
        sv[...] = r.integers(0, Q, size=sv.shape)
        e[...] = r.integers(0, Q, size=e.shape)
        o_plain, o_srv = pinned((n, k, 256)), pinned((n, k, 256))
        batch = (tk.MatvecBatch * 1)(tk.MatvecBatch(k, n, A.ctypes.data, sv.ctypes.data,
                                                    e.ctypes.data, o_plain.ctypes.data))
        tmpl.append(dict(k=k, n=n, A=A, s=sv, e=e, blk=blk, o_plain=o_plain, o_srv=o_srv, batch=batch,
                         ptrs=(A.ctypes.data, sv.ctypes.data, e.ctypes.data, o_srv.ctypes.data)))
    polys = np.array([t["n"] * t["k"] for t in tmpl])
    pc = time.perf_counter

    def plain_one(t):
        rc = L.tk_matvec_host(t["batch"], 1)
        if rc:
            raise tk.TKError(rc, L.tk_last_error().decode())

    for t in tmpl:                      # warm-up, reference outputs
        plain_one(t)
    t0 = pc()
    for t in tmpl:
        plain_one(t)
    service = (pc() - t0) / T
    cap = 1.0 / service

    def spin_until(x):
        while pc() < x:
            pass

    def pct(v, p):
        return float(np.percentile(np.asarray(v) * 1e6, p))

    mults = [float(x) for x in args.serve_rates.split(",")]
    # one arrival sequence per rate, shared by every arm
    runs = []
    for mult in mults:
        arr = np.cumsum(r.exponential(1.0 / (mult * cap), size=args.serve_requests))
        which = r.integers(0, T, size=args.serve_requests)
        runs.append((mult, arr, which, int(polys[which].sum())))
    points = [{"offered_x_plain_capacity": m, "offered_requests_per_s": m * cap,
               "requests": len(a), "polys": p} for m, a, _, p in runs]
    sampler = ClockSampler(0)
    sampler.start()
    # plain per-request launch, FIFO, with no server alive
    for pt, (mult, arr, which, tot_polys) in zip(points, runs):
        nreq = len(arr)
        lat = np.empty(nreq)
        base = pc() + 1e-3
        for i in range(nreq):
            ta = base + arr[i]
            spin_until(ta)
            plain_one(tmpl[which[i]])
            lat[i] = pc() - ta
        end = base + float(np.max(arr + lat))
        pt["plain"] = {"p50_us": pct(lat, 50), "p99_us": pct(lat, 99),
                       "polys_per_s": tot_polys / (end - base),
                       "requests_per_s": nreq / (end - base)}
    # each server arm alone: its device loop holds every SM while it runs
    arms = {"server": dict(zero_copy=False)}
    if args.serve_zero_copy:
        arms["server_zero_copy"] = dict(zero_copy=True)
    # server_arena: each rate's requests copied, in arrival order, back to back
    # into one pinned arena (as a receive ring would hold them), so that the
    # server's admission passes can take several requests' inputs in one copy
    msg_bytes = np.array([t["blk"].nbytes for t in tmpl], dtype=np.int64)
    arena = None
    if not args.serve_no_arena:
        need = max(int(msg_bytes[w].sum()) for _, _, w, _ in runs)
        arena = torch.empty(need // 2, dtype=torch.int16, pin_memory=True).numpy()
        arms["server_arena"] = dict(zero_copy=False)

    def request_ptrs(name, which):
        """Per request (A, s, e, out) addresses: the template's own buffers,
        or for the arena arm its message's place in the filled arena."""
        if name != "server_arena":
            return [tmpl[w]["ptrs"] for w in which]
        offs = np.concatenate([[0], np.cumsum(msg_bytes[which])[:-1]])
        out, base0 = [], arena.ctypes.data
        for o, w in zip(offs, which):
            t = tmpl[w]
            arena[o // 2:o // 2 + t["blk"].size] = t["blk"].ravel()
            a = base0 + int(o)
            sp = a + t["n"] * t["k"] * t["k"] * 512
            out.append((a, sp, sp + t["n"] * t["k"] * 512, t["ptrs"][3]))
        return out
    ticket = ctypes.c_uint64()
    stats = {}
    for name, kw in arms.items():
        srv = tk.Server(hbm_budget_bytes=1 << 30, max_inflight_requests=1024,
                        idle_exit_seconds=0.05, **kw)
        for t in tmpl:                  # warm-up
            a, b_, c, d = t["ptrs"]
            if L.tk_server_submit(srv._h, t["k"], t["n"], a, b_, c, d, ctypes.byref(ticket)):
                raise tk.TKError(1, "submit")
            srv.wait(ticket.value)
            srv.release(ticket.value)
        for t in tmpl:
            assert (t["o_srv"] == t["o_plain"]).all(), name
        st0 = srv.stats()
        for pt, (mult, arr, which, tot_polys) in zip(points, runs):
            nreq = len(arr)
            lag = np.empty(nreq)
            tickets = np.empty(nreq, dtype=np.uint64)
            ptrs = request_ptrs(name, which)
            base = pc() + 1e-3
            for i in range(nreq):
                ta = base + arr[i]
                spin_until(ta)
                t = tmpl[which[i]]
                a, b_, c, d = ptrs[i]
                rc = L.tk_server_submit(srv._h, t["k"], t["n"], a, b_, c, d,
                                        ctypes.byref(ticket))
                lag[i] = pc() - ta
                if rc:
                    raise tk.TKError(rc, "submit")
                tickets[i] = ticket.value
            slat = np.empty(nreq)
            for i in range(nreq):
                srv.wait(int(tickets[i]), timeout=60)
                slat[i] = lag[i] + srv.latency(int(tickets[i]))
                srv.release(int(tickets[i]))
            end = base + float(np.max(arr + slat))
            st = srv.stats()
            split = {f"mean_{x}_us": (st[f"{x}_ns"] - st0[f"{x}_ns"]) / 1e3 /
                     max(1, st["requests_done"] - st0["requests_done"])
                     for x in ("queue", "device", "return")}
            copies = (st["input_copies"] - st0["input_copies"]) / max(
                1, st["requests_done"] - st0["requests_done"])
            st0 = st
            pt[name] = {"p50_us": pct(slat, 50), "p99_us": pct(slat, 99),
                        "polys_per_s": tot_polys / (end - base),
                        "requests_per_s": nreq / (end - base),
                        "submit_lag_p99_us": pct(lag, 99),
                        "input_copies_per_request": copies, **split}
        stats[name] = srv.stats()
        srv.close()
    clocks = sampler.stop()
    exact = all((t["o_srv"] == t["o_plain"]).all() for t in tmpl)
    assert tk.device_status(0) == 0
    top = points[-1]
    print(json.dumps({
        "metric": "serving: p50/p99 request latency (us) and polys/s under Poisson arrivals, 1xB200",
        "value": top["server"]["polys_per_s"], "unit": "polys/s", "n_gpus": 1,
        "higher_is_better": True,
        "plain_service_us": service * 1e6, "plain_capacity_requests_per_s": cap,
        "points": points, "server_outputs_equal_plain": bool(exact),
        "server_stats": stats, "clocks": clocks,
        "config": {"workload": "requests of 1-64 matrix-vector jobs, k ~ U{2,3,4}, "
                               "coefficients uniform [0,q), pinned host buffers (A|s|e contiguous)",
                   "templates": T,
                   "plain_mode": ["pipeline", "fused", "tiled"][args.serve_plain_mode],
                   "server": "fused warp-per-job device loop",
                   "arms": {"server": "each request's A|s|e in its own pinned buffer",
                            "server_arena": "the same requests back to back in one pinned "
                                            "arena, in arrival order"}},
        "dtype": "int16", "data": "synthetic",
    }), flush=True)


def free_port() -> int:
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def launch_ranks(args) -> int:
    """--gpus N without a launcher: start N ranks (one per GPU) with
    torch.distributed.run on this node and return its exit status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
           f"--master-port={free_port()}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    world_env = os.environ.get("WORLD_SIZE")
    single = args.serve or args.forms or args.matvec or args.sweep or args.traffic
    if args.gpus < 1:
        sys.exit("bench.py: --gpus must be at least 1")
    if single and (args.gpus > 1 or (world_env is not None and int(world_env) > 1)):
        sys.exit("bench.py: --serve, --forms, --matvec, --sweep and --traffic run on one GPU "
                 "(--gpus 1)")
    if world_env is None and args.gpus > 1:
        sys.exit(launch_ranks(args))
    if world_env is not None and int(world_env) != args.gpus:
        sys.exit(f"bench.py: launched with WORLD_SIZE={world_env} but --gpus {args.gpus}; "
                 "pass --gpus equal to the number of ranks")
    if args.serve:
        run_serve(args)
    elif args.forms:
        run_forms(args)
    elif args.matvec:
        run_matvec(args)
    elif args.sweep:
        run_sweep(args)
    elif args.traffic:
        run_traffic(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
