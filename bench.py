"""Throughput benchmark of the lattice Monte Carlo hot path on B200.

Workload (one GPU): 3D q=3 Potts, 512^3 periodic, u8 states drawn uniformly
from the seed exactly as the reference's hot start does (RandRng +
Configuration::hot), beta = 0.5505, checkerboard heat bath on the reference
CPU stream (PCG64) -- bit-exact with the reference's CPU path.  One step =
one sweep of the lattice (134,217,728 site updates).  Under torchrun each rank
runs its own lattice (independent replicas, weak scaling; no collective on the
data path).

Prints one JSON line (rank 0).  ``--impl reference`` times the reference's
CPU algorithm (the C restatement in oracle/, single thread -- the reference
has no threading) on bounded samples of the same workload instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (512, 512, 512)
Q = 3
BETA = 0.5505
SEED = 20260718
WORKLOAD = ("3D q=3 Potts 512^3 periodic, checkerboard heat bath, beta=0.5505, PCG64 reference stream "
            "(bit-exact with the reference CPU path), uniform random u8 start from seed 20260718")
N_SITES = SHAPE[0] * SHAPE[1] * SHAPE[2]
BYTES_PER_UPDATE = 2  # each site read once and written once per sweep


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 6:
                self.samples.append((time.time(), parts))

    def stop(self, t0, t1):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        inside = [p for (t, p) in self.samples if t0 <= t <= t1] or [p for (_, p) in self.samples[-3:]]
        if not inside:
            return None
        sm = [float(p[0]) for p in inside if p[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for p in inside for i in range(4) if p[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(inside[0][1]) if inside[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(inside)}


def dist_setup(n_gpus):
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=None)
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, value, device):
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{device}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device):
    if pg is not None:
        import torch

        torch.cuda.synchronize(device)
        pg.barrier()


def run_product(args):
    import numpy as np
    import torch

    import plaquette_b200 as plq

    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    gpu = plq.Gpu.new(local)
    if gpu is None:
        raise RuntimeError("no CUDA device")
    seed = SEED + rank
    start, offset = plq.hot_start(seed, Q, N_SITES)

    # ---- device-resident throughput: K sweeps timed with CUDA events on the chain's stream
    desc = plq.make_desc(plq.POTTS, Q, SHAPE, plq.HEATBATH, beta=BETA, seed=seed, rng=plq.RNG_STREAM,
                         stream_offset=offset, sweeps_between=1, batch=plq.GPU_BATCH)
    chain = plq.GpuChain(gpu, desc, start)
    stream = torch.cuda.ExternalStream(chain.cuda_stream, device=f"cuda:{local}")
    chain.advance(args.warmup)
    chain.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg, local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = chain.launches
    t_wall0 = time.time()
    ev0.record(stream)
    chain.advance(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    t_wall1 = time.time()
    launches = chain.launches - launches0
    dev_ms = ev0.elapsed_time(ev1)
    clock_info = clocks.stop(t_wall0, t_wall1)
    chain.sync()
    dev_ms_max = max_over_ranks(pg, dev_ms, local)
    barrier(pg, local)

    sites_total = N_SITES * world * args.steps
    value = sites_total / (dev_ms_max * 1e6)  # site updates per ns
    ms_per_step = dev_ms_max / args.steps
    per_launch_ms = dev_ms / max(1, launches)
    alg_bytes = BYTES_PER_UPDATE * N_SITES
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic = profiled_traffic().get("fused3d_potts3_heatbath_stream_512", {}).get("dram_bytes_per_launch")

    # ---- end to end through the public API: pinned host start in, samples and final state out
    pinned = torch.empty(N_SITES, dtype=torch.uint8).pin_memory()
    pinned.numpy()[:] = start
    out_pinned = torch.empty(N_SITES, dtype=torch.uint8).pin_memory()
    barrier(pg, local)
    t0 = time.perf_counter()
    echain = plq.GpuChain(gpu, desc, pinned.numpy())
    _, prims = echain.next_batch(args.steps, states=False)
    rc = plq.lib().plq_chain_read(echain._h, out_pinned.data_ptr())
    plq.check(rc)
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(pg, t1 - t0, local)
    e2e_value = sites_total / (e2e_s * 1e9)
    echain.close()

    line = {
        "metric": "site updates/ns",
        "value": round(value, 3),
        "unit": "site updates/ns",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "sites_per_gpu": N_SITES, "step": "one sweep",
                   "l2": "inputs larger than L2 (two 134 MB state buffers, out-of-place sweep)",
                   "parallelism": f"independent lattice per GPU x{world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": alg_bytes, "kernel": "fused3d_kernel<3,true,true>"},
        "e2e": {"value": round(e2e_value, 3), "unit": "site updates/ns",
                "h2d_bytes_per_step": N_SITES / args.steps,
                "d2h_bytes_per_step": 8 * (1 + Q) + N_SITES / args.steps,
                "what": "chain create from pinned host start, K samples of one sweep each with device "
                        "primaries read back (GPU_BATCH at a time), final configuration read back"},
        "gpu_launches": launches,
        "clocks": clock_info,
    }
    if rank == 0 and args.cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    chain.close()
    if pg is not None:
        pg.destroy_process_group()


def cpu_baseline(seconds: float, steps: int = 1):
    """The reference CPU path (oracle restatement) on a bounded sample of the
    same workload: colour-0 heat-bath updates over a slice of the 512^3
    lattice, one thread (the reference has no threading)."""
    import numpy as np

    from oracle import oracle as o

    lat = o.Lattice(SHAPE)
    model = o.Model.potts(Q, 1.0)
    rng = o.PcgStream(SEED)
    cfg = o.hot_start(N_SITES, Q, rng)
    # warm-up slice
    o.local_site_slice(model, lat, cfg, o.HEATBATH, BETA, rng, 0, 0, 1 << 18)
    lo = 1 << 18
    chunk = 1 << 21
    total_updates, total_t = 0, 0.0
    times = []
    while total_t < seconds or len(times) < steps:
        t0 = time.perf_counter()
        n = o.local_site_slice(model, lat, cfg, o.HEATBATH, BETA, rng, 0, lo, lo + chunk)
        dt = time.perf_counter() - t0
        total_updates += n
        total_t += dt
        times.append(n / dt / 1e9)
        lo += chunk
        if lo + chunk > N_SITES:
            lo = 1 << 18
    del lat
    return {"value": round(total_updates / total_t / 1e9, 6), "unit": "site updates/ns", "cores": 1,
            "kind": "port",
            "sample": f"{total_updates} colour-0 heat-bath site updates of the 512^3 q=3 Potts lattice "
                      f"in slices of {chunk} sites ({total_t:.1f} s)"}


def run_reference(args):
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    if rank != 0:
        return
    import numpy as np

    from oracle import oracle as o

    lat = o.Lattice(SHAPE)
    model = o.Model.potts(Q, 1.0)
    rng = o.PcgStream(SEED)
    cfg = o.hot_start(N_SITES, Q, rng)
    chunk = 1 << 20  # site indices per step: one bounded sample of a sweep
    lo = 0

    def step():
        nonlocal lo
        n = o.local_site_slice(model, lat, cfg, o.HEATBATH, BETA, rng, 0, lo, lo + 2 * chunk)
        lo = (lo + 2 * chunk) % (N_SITES - 2 * chunk)
        return n

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    updates = sum(step() for _ in range(args.steps))
    dt = time.perf_counter() - t0
    value = updates / dt / 1e9
    line = {
        "metric": "site updates/ns", "value": round(value, 6), "unit": "site updates/ns", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "step": f"heat-bath updates of the colour-0 sites among {2 * chunk} "
                                                 "consecutive site indices (a bounded sample of one sweep)"},
        "cpu_baseline": {"value": round(value, 6), "unit": "site updates/ns", "cores": 1, "kind": "port",
                         "sample": f"{updates} site updates in {args.steps} steps"},
        "e2e": {"value": round(value, 6), "unit": "site updates/ns", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "product":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
