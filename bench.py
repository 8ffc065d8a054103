"""Throughput benchmark of the lattice Monte Carlo hot path on B200.

Default workload (one GPU): the batched ensemble -- 64 4D Z2 gauge lattices
(L 8/12/16/24 x 16, beta 0.40-0.48, link heat bath) beside 256 3D Ising
replicas in five parallel-tempering ladders (L 16-64, beta 0.20-0.24,
Metropolis, swaps every 10 sweeps), keyed stream, in one persistent
graph-captured launch per step, timed against the same sweeps with one
launch per lattice per colour pass.  One step = one tempering interval (10
sweeps of every member); the L2 cache is flushed between steps (the 49 MB
ensemble would otherwise stay resident).  The same run measures, as nested
records, the other configurations: 3D q=3 Potts 512^3 heat bath and 3D Ising
512^3 Metropolis (single-lattice HBM roofline), Swendsen-Wang 4096^2 over 500
sweeps, Wolff 128^3 over 10^5 single-cluster updates, and the serving loop at
the full job mix.  `--workload` runs one of them alone as the line.

Under torchrun each rank runs its own copy of the workload (independent
replicas, weak scaling; no collective on the data path; times are the max
over ranks).  `--gpus N` without torchrun launches N ranks itself.

Prints one JSON line (rank 0).  ``--impl reference`` times the reference's
CPU algorithm (the C restatement in oracle/) on bounded samples of the same
workload instead: the local sweeps on every host thread (one independent run
of site indices per thread; the reference itself is sequential), the cluster
moves on one thread.
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
SEED = 20260718
N_SITES = SHAPE[0] * SHAPE[1] * SHAPE[2]
BYTES_PER_UPDATE = 2  # each site read once and written once per sweep

# name -> (model, q, updater, rng, beta, description, dominant kernel, launches per sweep)
HIST_BINS = 1024

WORKLOADS = {
    "potts3-512-hb-stream": ("potts", 3, "heatbath", "stream", 0.5505,
                             "3D q=3 Potts 512^3 periodic, checkerboard heat bath, beta=0.5505, PCG64 reference "
                             "stream (bit-exact with the reference CPU path), uniform random u8 start from seed "
                             "20260718", "fused3d_kernel<3,true,true>", 1),
    "potts3-512-hb-keyed": ("potts", 3, "heatbath", "keyed", 0.5505,
                            "3D q=3 Potts 512^3 periodic, checkerboard heat bath, beta=0.5505, keyed reference GPU "
                            "stream, uniform random u8 start from seed 20260718", "fused3d_kernel<3,false,true>", 1),
    "ising-512-metro-keyed": ("ising", 2, "metropolis", "keyed", 0.2216544,
                              "3D Ising 512^3 periodic, checkerboard Metropolis, beta=0.2216544, keyed reference GPU "
                              "stream, uniform random start from seed 20260718", "fused3d_kernel<2,false,false>", 1),
    "ising-512-metro-stream": ("ising", 2, "metropolis", "stream", 0.2216544,
                               "3D Ising 512^3 periodic, checkerboard Metropolis, beta=0.2216544, PCG64 reference "
                               "stream (bit-exact with the reference CPU path; device-wide scan per colour pass), "
                               "uniform random start from seed 20260718", "scan_metro_kernel<3>", 2),
}


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

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        threading.Thread(target=self._read, daemon=True).start()
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


def dist_setup():
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, value, device):
    """Max of a per-rank time over all ranks (device None: a CPU tensor, for gloo)."""
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{device}" if device is not None else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, sites_per_rank, steps, max_ms):
    """Whole-job site updates per ns: every rank's sites over the slowest rank's time."""
    return sites_per_rank * world * steps / (max_ms * 1e6)


def nvtx_push(name):
    """An NVTX range (for profilers to select launches by); a no-op without NVTX."""
    try:
        import torch

        torch.cuda.nvtx.range_push(name)
    except Exception:
        pass


def nvtx_pop():
    try:
        import torch

        torch.cuda.nvtx.range_pop()
    except Exception:
        pass


def barrier(pg, device):
    if pg is not None:
        import torch

        torch.cuda.synchronize(device)
        pg.barrier()


def _desc(plq, w, seed, offset):
    model, q, upd, rng, beta = w[:5]
    return plq.make_desc({"potts": plq.POTTS, "ising": plq.ISING}[model], q, SHAPE,
                         {"heatbath": plq.HEATBATH, "metropolis": plq.METROPOLIS}[upd], beta=beta, seed=seed,
                         rng={"stream": plq.RNG_STREAM, "keyed": plq.RNG_KEYED}[rng], stream_offset=offset,
                         sweeps_between=1, batch=plq.GPU_BATCH)


class Ctx:
    """One rank's view of the job: rank numbers, the process group (None at
    N=1), its device and the library's context on it."""

    def __init__(self):
        import torch

        import plaquette_b200 as plq

        self.world, self.rank, self.local, self.pg = dist_setup()
        torch.cuda.set_device(self.local)
        self.gpu = plq.Gpu.new(self.local)
        if self.gpu is None:
            raise RuntimeError("no CUDA device")

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()


def traffic_record(name, kernel=None):
    """roofline.traffic from the committed ncu summary of this kernel (not
    measured in this run), with its source named; none when the summary is of
    another kernel than the one this run's path launches."""
    prof = profiled_traffic().get(name, {})
    if not prof or (kernel is not None and prof.get("kernel") != kernel):
        return None, None
    return prof.get("dram_bytes_per_launch"), (f"copied from {prof.get('summary')} (one ncu capture of this "
                                                f"kernel, {prof.get('captured', 'date in the summary')}); "
                                                "not measured in this run")


def measure_local(name, steps, warmup, ctx, e2e=True):
    """One 512^3 single-lattice workload: K sweeps timed with CUDA events on
    the chain's stream (inputs larger than L2), then, if asked, the same
    sweeps end to end through the public API."""
    import torch

    import plaquette_b200 as plq
    from plaquette_b200 import observables as obs

    w = WORKLOADS[name]
    world, local, pg, gpu = ctx.world, ctx.local, ctx.pg, ctx.gpu
    seed = SEED + ctx.rank
    start, offset = plq.hot_start(seed, w[1], N_SITES)

    desc = _desc(plq, w, seed, offset)
    chain = plq.GpuChain(gpu, desc, start)
    stream = torch.cuda.ExternalStream(chain.cuda_stream, device=f"cuda:{local}")
    chain.advance(warmup)
    chain.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg, local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = chain.launches
    t_wall0 = time.time()
    nvtx_push("timed")
    ev0.record(stream)
    chain.advance(steps)
    ev1.record(stream)
    nvtx_pop()
    ev1.synchronize()
    t_wall1 = time.time()
    launches = chain.launches - launches0
    dev_ms = ev0.elapsed_time(ev1)
    clock_info = clocks.stop(t_wall0, t_wall1)
    chain.sync()
    path = chain.path
    chain.close()
    dev_ms_max = max_over_ranks(pg, dev_ms, local)
    barrier(pg, local)

    sites_total = N_SITES * world * steps
    value = whole_job_rate(world, N_SITES, steps, dev_ms_max)
    kernel, per_sweep, l2_note = w[6], w[7], "inputs larger than L2 (134 MB state per lattice, two buffers for the " \
                                             "out-of-place sweep)"
    if path == "packed":
        # two pass launches per sweep on the 16.8 MB packed copy (L2-resident), the bytes packed and
        # unpacked once per advance call; their time is counted in the passes' average (conservative).
        # Each pass streams its colour's half of the 4 B/site first-hash array from HBM.
        kernel = f"packed_pass_kernel<3,{'true' if w[2] == 'heatbath' else 'false'},true>"
        per_sweep = 2
        l2_note = ("134 MB byte state read (packed) and written (unpacked) once per advance call; the sweeps run "
                   "on a 16.8 MB bit-packed copy that stays in L2 and stream each site's 4-byte first keyed hash "
                   "(537 MB, larger than L2) from HBM once per sweep")
    per_launch_ms = dev_ms / max(1, steps * per_sweep)
    alg_bytes = BYTES_PER_UPDATE * N_SITES // per_sweep  # per launch of the dominant kernel
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic, traffic_src = traffic_record(name, kernel)
    line = {
        "metric": "site updates/ns", "value": round(value, 3), "unit": "site updates/ns", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": round(dev_ms_max / steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": w[5], "name": name, "sites_per_gpu": N_SITES, "step": "one sweep",
                   "l2": l2_note,
                   "parallelism": f"independent lattice per GPU x{world}", "path": path},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_source": traffic_src,
                     "peak_source": peak_kind, "algorithmic_bytes_per_launch": alg_bytes, "kernel": kernel,
                     "note": "instruction-issue bound: the reference's per-site RNG (a 128-bit LCG step or "
                             "two 32-bit hashes per draw) costs more issue slots than HBM allows at 2 B/update"},
        "gpu_launches": launches,
        "clocks": clock_info,
    }
    if not e2e:
        return line

    # end to end through the public API: pinned host start in, samples and final state out
    pinned = torch.empty(N_SITES, dtype=torch.uint8).pin_memory()
    pinned.numpy()[:] = start
    out_pinned = torch.empty(N_SITES, dtype=torch.uint8).pin_memory()
    barrier(pg, local)
    t0 = time.perf_counter()
    echain = plq.GpuChain(gpu, desc, pinned.numpy())
    _, prims = echain.next_batch(steps, states=False)
    plq.check(plq.lib().plq_chain_read(echain._h, out_pinned.data_ptr()))
    # per-sweep energy and order-parameter histograms (1024 bins) from the exact primaries
    model = obs.POTTS if w[0] == "potts" else obs.ISING
    ser = obs.series(model, prims, N_SITES)
    hist_e = obs.histogram(ser["e"], HIST_BINS, -3.0, 3.0)
    hist_m = obs.histogram(ser["m"], HIST_BINS, 0.0, 1.0)
    t1 = time.perf_counter()
    assert int(hist_e.sum()) == int(hist_m.sum()) == steps
    e2e_s = max_over_ranks(pg, t1 - t0, local)
    n_prim = len(prims[0])
    echain.close()
    line["e2e"] = {"value": round(sites_total / (e2e_s * 1e9), 3), "unit": "site updates/ns",
                   "h2d_bytes_per_step": N_SITES / steps,
                   "d2h_bytes_per_step": 8 * n_prim + N_SITES / steps,
                   "what": "chain create from a pinned host start, K samples of one sweep each with their device "
                           "primaries read back, per-sweep E/N and order-parameter histograms "
                           f"({HIST_BINS} bins), final configuration read back"}
    return line


def run_product(args):
    ctx = Ctx()
    line = measure_local(args.workload, args.steps, args.warmup, ctx)
    if ctx.rank == 0 and args.cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload, args.cpu_seconds)
    if ctx.rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def _oracle_setup(name):
    from oracle import oracle as o

    w = WORKLOADS[name]
    lat = o.Lattice(SHAPE)
    model = o.Model.potts(w[1], 1.0) if w[0] == "potts" else o.Model.ising(1.0, 0.0)
    kernel = o.HEATBATH if w[2] == "heatbath" else o.METROPOLIS
    rng = o.PcgStream(SEED)
    cfg = o.hot_start(N_SITES, w[1], rng)
    return o, w, lat, model, kernel, rng, cfg


def _host_threads() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return max(1, os.cpu_count() or 1)


class _SliceRunner:
    """The reference CPU path (the oracle's restatement of LocalUpdate's
    checkerboard) on every host core: thread t updates the colour-0 sites of
    its own run of site indices with its own PCG stream.  Colour-0 updates read
    only colour-1 neighbours, so the threads never touch each other's inputs;
    the reference itself is sequential, so this is T independent samples of
    its work side by side (the oracle releases the GIL inside each call)."""

    def __init__(self, name: str, threads: int, span: int):
        from concurrent.futures import ThreadPoolExecutor

        self.o, self.w, self.lat, self.model, self.kernel, _, self.cfg = _oracle_setup(name)
        self.threads, self.span = threads, span
        self.rngs = [self.o.PcgStream(SEED + 1 + t) for t in range(threads)]
        self.pool = ThreadPoolExecutor(threads)
        self.lo = 0

    def _one(self, t: int, lo: int) -> int:
        a = lo + t * self.span
        return self.o.local_site_slice(self.model, self.lat, self.cfg, self.kernel, self.w[4], self.rngs[t], 0, a,
                                       a + self.span)

    def step(self) -> int:
        """One step: every thread updates its run; returns the site updates made."""
        lo = self.lo
        n = sum(self.pool.map(lambda t: self._one(t, lo), range(self.threads)))
        self.lo = (lo + self.threads * self.span) % (N_SITES - self.threads * self.span)
        return n

    def close(self):
        self.pool.shutdown()


def cpu_baseline(name: str, seconds: float):
    """The reference CPU path on a bounded sample of the same workload, on all
    host cores (one independent run of site indices per thread)."""
    threads = _host_threads()
    r = _SliceRunner(name, threads, 1 << 19)
    r.step()  # warm-up
    total_updates, total_t = 0, 0.0
    while total_t < seconds:
        t0 = time.perf_counter()
        total_updates += r.step()
        total_t += time.perf_counter() - t0
    r.close()
    return {"value": round(total_updates / total_t / 1e9, 6), "unit": "site updates/ns", "cores": threads,
            "kind": "port",
            "sample": f"{total_updates} colour-0 site updates of the {name} workload, {threads} threads each on its "
                      f"own run of {1 << 19} site indices per step ({total_t:.1f} s)"}


def run_reference(args):
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    if rank != 0:
        return
    threads = _host_threads()
    span = 1 << 19  # site indices per thread per step: a bounded sample of one sweep
    r = _SliceRunner(args.workload, threads, span)
    w = r.w
    for _ in range(args.warmup):
        r.step()
    t0 = time.perf_counter()
    updates = sum(r.step() for _ in range(args.steps))
    dt = time.perf_counter() - t0
    r.close()
    value = updates / dt / 1e9
    line = {
        "metric": "site updates/ns", "value": round(value, 6), "unit": "site updates/ns", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": w[5], "name": args.workload, "sites_per_gpu": N_SITES,
                   "step": f"updates of the colour-0 sites among {threads} x {span} site indices, one run per host "
                           "thread (a bounded sample of one sweep)"},
        "cpu_baseline": {"value": round(value, 6), "unit": "site updates/ns", "cores": threads, "kind": "port",
                         "sample": f"{updates} site updates in {args.steps} steps on {threads} threads"},
        "e2e": {"value": round(value, 6), "unit": "site updates/ns", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


ENSEMBLE_WORKLOAD = "ensemble-config4"
PT_EVERY = 10           # tempering interval: one bench step
L2_FLUSH_BYTES = 256 << 20  # written between timed steps: twice the 126 MB L2


def timed_steps(stream, fn, steps, sweeps_per_step, flush):
    """`steps` calls of fn(sweeps_per_step), each bracketed by CUDA events on
    `stream`, with an L2 flush (a 256 MB write on the same stream) before
    each, outside the events.  Returns the summed device milliseconds."""
    import torch

    pairs = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nvtx_push("timed")  # profilers select the timed launches by this range
        fn(sweeps_per_step)
        nvtx_pop()
        e1.record(stream)
        pairs.append((e0, e1))
    pairs[-1][1].synchronize()
    return sum(e0.elapsed_time(e1) for e0, e1 in pairs)


def measure_ensemble(steps, warmup, ctx):
    """The batched ensemble: one persistent graph-captured launch per step
    (10 sweeps of every member, one tempering phase), timed against the same
    sweeps with one launch per lattice per colour pass."""
    import numpy as np
    import torch

    import plaquette_b200 as plq
    from plaquette_b200.ensemble import batched_workload_spec, build_ensemble, tune_entries

    world, local, pg, gpu = ctx.world, ctx.local, ctx.pg, ctx.gpu
    seed = SEED + ctx.rank
    descs, starts, ladders = batched_workload_spec(seed)
    n_vars = int(sum(len(x) for x in starts))
    ens = build_ensemble(gpu, descs, starts, ladders, seed, pt_every=PT_EVERY)
    # the autotuner: a work-item shape per member shape, then the launch shape (state restored after)
    t_tune = time.perf_counter()
    tuned_r, tuned_c, tuned_ms = ens.tune(PT_EVERY)
    tuning = {"launch": {"ranks_per_thread": tuned_r, "ctas_per_sm": tuned_c,
                         "ms_per_sweep": round(tuned_ms, 5)},
              "shapes": tune_entries(), "seconds": round(time.perf_counter() - t_tune, 2)}
    stream = torch.cuda.ExternalStream(ens.cuda_stream, device=f"cuda:{local}")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(warmup):
        ens.advance(PT_EVERY)
    ens.sync()

    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg, local)
    launches0 = ens.launches
    t_wall0 = time.time()
    batched_ms = timed_steps(stream, ens.advance, steps, PT_EVERY, flush)
    t_wall1 = time.time()
    launches = ens.launches - launches0
    clock_info = clocks.stop(t_wall0, t_wall1)
    k_unb = min(steps, 5)
    unbatched_ms = timed_steps(stream, ens.advance_unbatched, k_unb, PT_EVERY, flush)
    batched_ms_max = max_over_ranks(pg, batched_ms, local)
    unbatched_ms_max = max_over_ranks(pg, unbatched_ms, local)

    # identical observables: a second ensemble from the same seeds, every sweep per-lattice
    ref = build_ensemble(gpu, descs, starts, ladders, seed, pt_every=PT_EVERY)
    ref.set_config(tuned_r, tuned_c)
    ref.advance_unbatched((warmup + steps + k_unb) * PT_EVERY)
    same = all(np.array_equal(a, b) for a, b in zip(ens.primaries_all(), ref.primaries_all())) and \
        np.array_equal(ens.betas(), ref.betas())
    ref.close()
    ens.close()

    # end to end through the public API: starts from pinned host memory in; after every step
    # every member's primaries and beta out
    pinned = torch.empty(n_vars, dtype=torch.uint8).pin_memory()
    views, off = [], 0
    for st in starts:
        v = pinned.numpy()[off:off + len(st)]
        v[:] = st
        views.append(v)
        off += len(st)
    barrier(pg, local)
    t0 = time.perf_counter()
    e2 = build_ensemble(gpu, descs, views, ladders, seed, pt_every=PT_EVERY)
    e2.set_config(tuned_r, tuned_c)
    t_made = time.perf_counter()
    n_prim = 0
    for _ in range(steps):
        e2.advance(PT_EVERY)
        prims = e2.primaries_all()
        betas = e2.betas()
        n_prim = sum(len(p) for p in prims)
    t1 = time.perf_counter()
    assert len(betas) == e2.n
    e2.close()
    e2e_s = max_over_ranks(pg, t1 - t0, local)

    updates = n_vars * world * steps * PT_EVERY
    value = updates / (batched_ms_max * 1e-3) / 1e9
    unb_value = n_vars * world * k_unb * PT_EVERY / (unbatched_ms_max * 1e-3) / 1e9
    alg_bytes = BYTES_PER_UPDATE * n_vars * PT_EVERY  # per launch (one step)
    achieved = alg_bytes * steps / (batched_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic, traffic_src = traffic_record(ENSEMBLE_WORKLOAD)
    return {
        "metric": "site updates/ns", "value": round(value, 3), "unit": "site updates/ns", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": round(batched_ms_max / steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "64 4D Z2 gauge lattices (L 8/12/16/24 x 16, beta 0.40-0.48, link heat bath) + "
                               "256 3D Ising replicas (L 16-64, five ladders, beta 0.20-0.24 geometric, "
                               "Metropolis, tempering swaps every 10 sweeps), keyed stream, hot starts",
                   "name": ENSEMBLE_WORKLOAD, "members": len(descs), "variables": n_vars,
                   "step": f"one tempering interval: {PT_EVERY} sweeps of every member and one swap phase, one "
                           "graph-captured persistent launch",
                   "l2": "L2 flushed between timed steps (a 256 MB write outside the timed events); the 49 MB "
                         "ensemble is L2-resident within a step",
                   "parallelism": f"independent ensemble per GPU x{world}"},
        "per_lattice_launches": {"value": round(unb_value, 3), "steps": k_unb,
                                 "ms_per_step": round(unbatched_ms_max / k_unb, 5),
                                 "what": "the same sweeps and swaps with one launch per lattice per colour pass"},
        "batched_over_per_lattice": round(value / unb_value, 2),
        "identical_observables": bool(same),
        "tuning": tuning,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_source": traffic_src,
                     "peak_source": peak_kind, "algorithmic_bytes_per_launch": alg_bytes,
                     "kernel": "ensemble_kernel",
                     "note": "2 B per variable update; the ensemble (49 MB) is read from HBM once per step and "
                             "then served from L2"},
        "e2e": {"value": round(updates / (e2e_s * 1e9), 3), "unit": "site updates/ns",
                "h2d_bytes_per_step": n_vars / steps,
                "d2h_bytes_per_step": 8 * n_prim + 8 * len(descs),
                "create_ms": round((t_made - t0) * 1e3, 2), "steps_ms": round((t1 - t_made) * 1e3, 2),
                "what": "ensemble create from pinned host starts, then K steps each followed by every member's "
                        "primaries and beta read back"},
        "gpu_launches": launches,
        "clocks": clock_info,
    }


def measure_serving(rate, n_jobs, ctx):
    """The serving loop at one Poisson arrival rate over the full job mix
    (100-5000 sweeps per job)."""
    from plaquette_b200.serving import run_poisson

    barrier(ctx.pg, ctx.local)
    r = run_poisson(ctx.gpu, rate, n_jobs, seed=int(rate) + 7 * ctx.rank, sweeps_scale=1.0)
    p99 = max_over_ranks(ctx.pg, r["p99_ms"], ctx.local)
    return {"metric": "job p99 ms", "value": round(p99, 2), "unit": "ms", "higher_is_better": False,
            "p50_ms": round(r["p50_ms"], 2), "mean_ms": round(r["mean_ms"], 2),
            "rate_jobs_per_s": rate, "jobs": n_jobs,
            "site_updates_per_ns_busy": round(r["site_updates_per_ns_busy"], 2), "ticks": r["ticks"],
            "wall_s": round(r["wall_s"], 2),
            "config": {"workload": "Poisson arrivals of mixed jobs: 50% 2D/3D Ising Metropolis (2D L 32-1024, "
                                   "3D L 16-256), 30% 3D Potts q=3/4 heat bath, 20% 4D Z2 gauge heat bath (L 8-24), "
                                   "beta within 2% of the transition, 100-5000 sweeps each (full range), keyed"}}


RECORD_WORKLOADS = ("potts3-512-hb-stream", "ising-512-metro-keyed", "ising-512-metro-stream",
                    "sw-4096-keyed", "sw-4096-stream", "wolff-128-keyed")


def _record(line):
    keep = ("metric", "value", "unit", "ms_per_step", "steps", "higher_is_better", "roofline", "e2e",
            "size_histogram_log2", "gpu_launches", "clocks")
    out = {k: line[k] for k in keep if k in line}
    out["workload"] = line["config"]["workload"]
    return out


def run_ensemble(args):
    ctx = Ctx()
    line = measure_ensemble(args.steps, args.warmup, ctx)
    if args.records:
        records = {}
        for name in RECORD_WORKLOADS:
            try:
                if name in WORKLOADS:
                    rec = measure_local(name, args.steps, args.warmup, ctx, e2e=(name == "potts3-512-hb-stream"))
                else:
                    steps, _ = CLUSTER_RECORD_STEPS[name]
                    rec = measure_cluster(name, steps, 3, ctx, e2e=False)
                records[name] = _record(rec)
            except Exception as exc:  # one failing record must not hide the others
                records[name] = {"error": f"{type(exc).__name__}: {exc}"}
        try:
            records["serving-10-jobs-per-s"] = measure_serving(10.0, 60, ctx)
        except Exception as exc:
            records["serving-10-jobs-per-s"] = {"error": f"{type(exc).__name__}: {exc}"}
        line["records"] = records
    if ctx.rank == 0 and args.cpu_baseline:
        cv, threads, n_members, _, dt_c = ensemble_cpu_sample(steps=6, warmup=1)
        line["cpu_baseline"] = {"value": round(cv, 6), "unit": "site updates/ns", "cores": threads, "kind": "port",
                                "sample": f"6 sweeps of all {n_members} members on {threads} threads "
                                          f"({dt_c:.1f} s; tempering swaps left out)"}
    if ctx.rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


CLUSTER_WORKLOADS = {
    # name: (extent, rng, shape, beta, what)
    "sw-4096-keyed": ("all", "keyed", (4096, 4096), 0.4406868,
                      "2D Ising 4096^2 periodic Swendsen-Wang, beta=0.4406868, p=1-exp(-2 beta), keyed reference "
                      "GPU stream, uniform random start"),
    "sw-4096-stream": ("all", "stream", (4096, 4096), 0.4406868,
                       "2D Ising 4096^2 periodic Swendsen-Wang, beta=0.4406868, PCG64 reference stream (bit-exact "
                       "with the reference CPU ClusterUpdate), uniform random start"),
    "wolff-128-keyed": ("seeded", "keyed", (128, 128, 128), 0.2216544,
                        "3D Ising 128^3 periodic Wolff (keyed seed site, frontier BFS), beta=0.2216544, uniform "
                        "random start"),
}


# record steps: (steps, units per step) -- SW over the configuration's 500 sweeps, Wolff over 10^5 updates
CLUSTER_RECORD_STEPS = {"sw-4096-keyed": (500, 1), "sw-4096-stream": (500, 1), "wolff-128-keyed": (100, 1000)}


def measure_cluster(name, steps, warmup, ctx, e2e=True):
    """Cluster moves: Swendsen-Wang sweeps/s (labels, size histogram each
    sweep available) or Wolff single-cluster updates/s."""
    import numpy as np
    import torch

    import plaquette_b200 as plq

    extent, rng_name, shape, beta, what = CLUSTER_WORKLOADS[name]
    world, local, pg, gpu = ctx.world, ctx.local, ctx.pg, ctx.gpu
    seed = SEED + ctx.rank
    n = int(np.prod(shape))
    start, offset = plq.hot_start(seed, 2, n)
    rng = plq.RNG_STREAM if rng_name == "stream" else plq.RNG_KEYED
    ext = plq.EXTENT_ALL if extent == "all" else plq.EXTENT_SEEDED
    relabel = plq.RELABEL_REDRAW if extent == "all" else plq.RELABEL_FORCED
    wolff = extent == "seeded"
    per_step = 1000 if wolff else 1  # Wolff: one step = 1000 single-cluster updates

    def make(st):
        d = plq.make_desc(plq.ISING, 2, shape, plq.CLUSTER, beta=beta, seed=seed, rng=rng, stream_offset=offset,
                          sweeps_between=per_step, batch=1, extent=ext, relabel=relabel)
        return plq.GpuClusterChain(gpu, d, st)

    chain = make(start)
    stream = torch.cuda.ExternalStream(chain.cuda_stream, device=f"cuda:{local}")
    chain.advance(warmup * per_step)
    chain.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg, local)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = chain.launches
    t_wall0 = time.time()
    ev0.record(stream)
    nvtx_push("timed")
    chain.advance(steps * per_step)
    nvtx_pop()
    ev1.record(stream)
    ev1.synchronize()
    t_wall1 = time.time()
    chain.sync()
    launches = chain.launches - launches0
    clock_info = clocks.stop(t_wall0, t_wall1)
    dev_ms = max_over_ranks(pg, ev0.elapsed_time(ev1), local)
    units = steps * per_step * world
    value = units / (dev_ms * 1e-3)
    hist = chain.size_histogram(32)
    chain.close()
    unit = "cluster updates/s" if wolff else "SW sweeps/s"
    alg = 10.5 * n if not wolff else None  # SW: spins r+w, bond bits r+w, labels w+r (bytes per sweep)
    peak, peak_kind = measured_peak_hbm()
    line = {
        "metric": unit, "value": round(value, 2), "unit": unit, "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": round(dev_ms / steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": what, "name": name, "sites": n,
                   "step": "1000 single-cluster updates" if wolff else "one Swendsen-Wang sweep",
                   "l2": "state, bonds and labels (16.8 M sites: 101 MB) stream through L2 every sweep" if not wolff
                   else "cluster work only; the 2.1 MB lattice stays in L2",
                   "parallelism": f"independent lattice per GPU x{world}"},
        "roofline": ({"bound": "hbm", "achieved": round(alg * steps / (dev_ms * 1e-3) / 1e9, 1),
                      "peak": peak, "unit": "GB/s",
                      "frac": round(alg * steps / (dev_ms * 1e-3) / 1e9 / peak, 4),
                      "traffic": None, "peak_source": peak_kind,
                      "algorithmic_bytes_per_launch": alg,
                      "kernel": "bonds + tile union-find + boundary unions + relabel",
                      "note": "10.5 B/site per sweep algorithmic minimum"} if not wolff else
                     {"bound": "latency", "achieved": None, "peak": None, "unit": None, "frac": None,
                      "traffic": None, "note": "frontier BFS: work proportional to the cluster, not the lattice"}),
        "size_histogram_log2": [int(x) for x in hist[:24]],
        "gpu_launches": launches,
        "clocks": clock_info,
    }
    if not e2e:
        return line

    # end to end: chain from a pinned host start, K steps, size histogram and final configuration back
    pinned = torch.empty(n, dtype=torch.uint8).pin_memory()
    pinned.numpy()[:] = start
    out_pinned = torch.empty(n, dtype=torch.uint8).pin_memory()
    barrier(pg, local)
    t0 = time.perf_counter()
    ec = make(pinned.numpy())
    ec.advance(steps * per_step)
    ec.size_histogram(32)
    plq.check(plq.lib().plq_chain_read(ec._h, out_pinned.data_ptr()))
    t1 = time.perf_counter()
    ec.close()
    e2e_s = max_over_ranks(pg, t1 - t0, local)
    line["e2e"] = {"value": round(units / e2e_s, 2), "unit": unit, "h2d_bytes_per_step": n / steps,
                   "d2h_bytes_per_step": (n + 8 * 32) / steps,
                   "what": "chain create from a pinned host start, K steps, cluster-size histogram and final "
                           "configuration read back"}
    return line


def run_cluster(args):
    ctx = Ctx()
    line = measure_cluster(args.workload, args.steps, args.warmup, ctx)
    if ctx.rank == 0 and args.cpu_baseline:
        units_c, dt_c, sample = cluster_cpu_sample(args.workload, args.cpu_seconds)
        line["cpu_baseline"] = {"value": round(units_c / dt_c, 4), "unit": line["unit"], "cores": 1,
                                "kind": "port", "sample": sample}
    if ctx.rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def cluster_cpu_sample(name: str, seconds: float, warmup: int = 0, max_units: int = 1 << 30):
    """The oracle's restatement of the reference cluster move on one host
    thread (the reference is sequential), on the workload's lattice from the
    same start: Swendsen-Wang sweeps, or keyed Wolff updates (the reference
    GPU's seeded decomposition filter), for about `seconds` after `warmup`
    untimed ones.  Returns (units, seconds, description)."""
    from oracle import oracle
    import plaquette_b200 as plq

    extent, rng_name, shape, beta, what = CLUSTER_WORKLOADS[name]
    lat = oracle.Lattice(shape)
    model = oracle.Model.ising(1.0)
    start, off = plq.hot_start(SEED, 2, lat.n_sites)
    state = start.copy()
    ext = oracle.ALL if extent == "all" else oracle.SEEDED
    relabel = oracle.REDRAW if extent == "all" else oracle.FORCED
    if rng_name == "stream":
        r = oracle.PcgStream(SEED)
        r.advance(off)

        def step(k):
            oracle.cluster_sweep(model, lat, state, ext, relabel, beta, r)
    else:
        s32 = oracle.fold_seed(SEED)

        def step(k):
            oracle.keyed_cluster_sweep(model, lat, state, ext, relabel, beta, s32, k)
    for k in range(warmup):
        step(k)
    done = 0
    t0 = time.perf_counter()
    while done < max_units and (done == 0 or time.perf_counter() - t0 < seconds):
        step(warmup + done)
        done += 1
    dt = time.perf_counter() - t0
    what_unit = "sweeps" if extent == "all" else "single-cluster updates"
    return done, dt, f"{done} {what_unit} of the {'x'.join(map(str, shape))} lattice on one host thread"


def ensemble_cpu_sample(steps: int, warmup: int):
    """The batched-ensemble members on the host: the reference runs one chain
    at a time, so each member's keyed sweep is the oracle's restatement of the
    reference GPU checkerboard, the members spread over every host thread (one
    member per thread at a time; lattices of one shape share their neighbour
    and staple tables).  A step is one sweep of every member; the tempering
    swaps (every 10 sweeps, a few hundred energy comparisons) are left out.
    Returns (site updates/ns, threads, members, variables, seconds)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle
    import plaquette_b200 as plq
    from plaquette_b200.ensemble import batched_workload_spec

    descs, starts, _ = batched_workload_spec()
    lattices, members = {}, []
    for d, start in zip(descs, starts):
        shape = tuple(int(d.shape[i]) for i in range(d.d))
        gauge = d.model == plq.GAUGE
        if (shape, gauge) not in lattices:
            lattices[(shape, gauge)] = oracle.Lattice(shape, staples=gauge)
        model = oracle.Model.gauge(d.j) if gauge else oracle.Model.ising(d.j, d.h)
        kernel = oracle.HEATBATH if d.updater == plq.HEATBATH else oracle.METROPOLIS
        members.append((model, lattices[(shape, gauge)], start.copy(), kernel, d.beta, oracle.fold_seed(d.seed)))
    n_vars = sum(len(m[2]) for m in members)
    threads = _host_threads()
    # largest members first, so the pool ends evenly
    order = sorted(range(len(members)), key=lambda i: -len(members[i][2]))

    def one(i, k):
        model, lat, cfg, kernel, beta, s32 = members[i]
        oracle.keyed_local_sweep(model, lat, cfg, kernel, beta, s32, k)

    with ThreadPoolExecutor(threads) as ex:
        for k in range(warmup):
            list(ex.map(lambda i: one(i, k), order))
        t0 = time.perf_counter()
        for k in range(warmup, warmup + steps):
            list(ex.map(lambda i: one(i, k), order))
        dt = time.perf_counter() - t0
    return n_vars * steps / dt / 1e9, threads, len(members), n_vars, dt


def run_reference_ensemble(args):
    """The reference arm of the batched ensemble (ensemble_cpu_sample)."""
    world = _env_int("WORLD_SIZE", 1)
    if _env_int("RANK", 0) != 0:
        return
    value, threads, n_members, n_vars, dt = ensemble_cpu_sample(args.steps, args.warmup)
    unit = "site updates/ns"
    line = {
        "metric": unit, "value": round(value, 6), "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": "the batched-ensemble members (64 4D Z2 gauge lattices + 256 3D Ising replicas), "
                               "one keyed sweep each per step", "name": ENSEMBLE_WORKLOAD,
                   "members": n_members, "variables": n_vars,
                   "step": "one sweep of every member (tempering swaps left out)"},
        "cpu_baseline": {"value": round(value, 6), "unit": unit, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} sweeps of all {n_members} members on {threads} threads"},
        "e2e": {"value": round(value, 6), "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_cluster(args):
    """The reference arm of a cluster workload: the oracle's cluster move on
    one host thread, `steps` sweeps or updates after `warmup` untimed ones."""
    world = _env_int("WORLD_SIZE", 1)
    if _env_int("RANK", 0) != 0:
        return
    extent = CLUSTER_WORKLOADS[args.workload][0]
    unit = "cluster updates/s" if extent == "seeded" else "SW sweeps/s"
    units, dt, sample = cluster_cpu_sample(args.workload, float("inf"), warmup=args.warmup, max_units=args.steps)
    value = units / dt
    line = {
        "metric": unit, "value": round(value, 4), "unit": unit, "n_gpus": world, "steps": units,
        "warmup": args.warmup, "ms_per_step": round(dt / units * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": CLUSTER_WORKLOADS[args.workload][4], "name": args.workload,
                   "step": "one sweep" if extent == "all" else "one single-cluster update"},
        "cpu_baseline": {"value": round(value, 4), "unit": unit, "cores": 1, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 4), "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def spawn_ranks(n: int) -> int:
    """`bench.py --gpus N` outside torchrun: relaunch this command as N ranks
    on this node (127.0.0.1 rendezvous) and return their exit status."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--workload", default=ENSEMBLE_WORKLOAD,
                    choices=[ENSEMBLE_WORKLOAD] + sorted(WORKLOADS) + sorted(CLUSTER_WORKLOADS))
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-records", dest="records", action="store_false",
                    help="ensemble workload: skip the nested records of the other configurations")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    if args.warmup < 3 and args.impl == "product":
        args.warmup = 3
    if args.impl == "reference" and args.workload in CLUSTER_WORKLOADS:
        run_reference_cluster(args)
    elif args.impl == "reference" and args.workload == ENSEMBLE_WORKLOAD:
        run_reference_ensemble(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == ENSEMBLE_WORKLOAD:
        run_ensemble(args)
    elif args.workload in CLUSTER_WORKLOADS:
        run_cluster(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
