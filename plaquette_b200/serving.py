"""Serving: a continuous-batching request loop for simulation jobs.

``Server`` wraps the ``plq_server_*`` entry points of include/plaquette.h.
Jobs (a chain descriptor, a start configuration, a number of sweeps) are
admitted by device-memory footprint, stay resident on the device, and share
one persistent launch per tick with every other running job.

``python -m plaquette_b200.serving`` runs the Poisson-arrival benchmark: a
mix of 50 % Ising (2D L ~ U[32,1024], 3D L ~ U[16,256]), 30 % 3D Potts
q in {3,4}, 20 % 4D Z2 gauge L ~ U[8,24], beta within +-2 % of the model's
transition, sweeps ~ U[100,5000]; it reports p50/p99 job latency and the
aggregate site updates/ns per arrival rate.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import (GAUGE, HEATBATH, ISING, METROPOLIS, POTTS, RNG_KEYED, ChainDesc, Gpu, check, extra_signatures,
               lib, make_desc)

JOB_QUEUED, JOB_ACTIVE, JOB_DONE, JOB_FAILED, JOB_CANCELLED = range(5)

_P = C.POINTER
extra_signatures({
    "plq_server_create": ([C.c_void_p, C.c_uint64, C.c_int32, C.c_double, _P(C.c_void_p)], C.c_int),
    "plq_server_submit": ([C.c_void_p, _P(ChainDesc), C.c_void_p, C.c_uint64, C.c_int32, _P(C.c_int64)], C.c_int),
    "plq_server_wait": ([C.c_void_p, C.c_int64, C.c_double, _P(C.c_int32)], C.c_int),
    "plq_server_cancel": ([C.c_void_p, C.c_int64], C.c_int),
    "plq_server_result": ([C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "plq_server_release": ([C.c_void_p, C.c_int64], C.c_int),
    "plq_server_stats": ([C.c_void_p, C.c_void_p], C.c_int),
    "plq_server_destroy": ([C.c_void_p], None),
})

# Transition couplings the job generator centres beta on.
BETA_C = {("ising", 2): 0.4406868, ("ising", 3): 0.2216544, ("potts", 3): 0.5505, ("potts", 4): 0.6286,
          ("gauge", 4): 0.4407}


class Server:
    def __init__(self, gpu: Gpu, budget_bytes: int = 0, max_slots: int = 64, tick_ms: float = 10.0):
        self.gpu = gpu
        self._h = C.c_void_p()
        # bound now: at interpreter exit the module's globals may already be gone
        self._destroy = lib().plq_server_destroy
        check(lib().plq_server_create(gpu._h, budget_bytes, max_slots, tick_ms, C.byref(self._h)))
        self._jobs = {}

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    __del__ = close

    def submit(self, desc: ChainDesc, start: np.ndarray | None, sweeps: int, want_states: bool = False) -> int:
        jid = C.c_int64()
        ptr = None
        if start is not None:
            start = np.ascontiguousarray(start, dtype=np.uint8)
            ptr = start.ctypes.data
        check(lib().plq_server_submit(self._h, C.byref(desc), ptr, sweeps, int(want_states), C.byref(jid)))
        n = int(np.prod([desc.shape[i] for i in range(desc.d)]))
        self._jobs[jid.value] = (n * desc.d if desc.model == GAUGE else n, desc)
        return jid.value

    def submit_run(self, spec, want_states: bool = False) -> int:
        """Submit a parsed run configuration (runspec.parse): its start
        configuration and all its sweeps, thermalisation included."""
        from .runspec import start_configuration

        start, offset = start_configuration(spec)
        spec.desc.stream_offset = offset
        return self.submit(spec.desc, start, spec.total_sweeps, want_states)

    def wait(self, job: int, timeout_s: float = -1.0) -> int:
        st = C.c_int32()
        check(lib().plq_server_wait(self._h, job, timeout_s, C.byref(st)))
        return st.value

    def cancel(self, job: int) -> None:
        check(lib().plq_server_cancel(self._h, job))

    def result(self, job: int, states: bool = False):
        n_vars, desc = self._jobs[job]
        out = np.empty(n_vars, dtype=np.uint8) if states else None
        prim = np.zeros(66, dtype=np.int64)
        timing = np.zeros(2, dtype=np.float64)
        check(lib().plq_server_result(self._h, job, out.ctypes.data if states else None, prim.ctypes.data,
                                      timing.ctypes.data))
        n_prim = {ISING: 2, POTTS: 1 + desc.q, GAUGE: 1}[desc.model]
        return out, prim[:n_prim].copy(), {"queue_ms": float(timing[0]), "latency_ms": float(timing[1])}

    def release(self, job: int) -> None:
        check(lib().plq_server_release(self._h, job))
        self._jobs.pop(job, None)

    def stats(self) -> dict:
        out = np.zeros(8, dtype=np.float64)
        rc = lib().plq_server_stats(self._h, out.ctypes.data)
        keys = ["completed", "p50_ms", "p99_ms", "site_updates_per_ns", "ticks", "queued", "running", "device_bytes"]
        d = dict(zip(keys, out.tolist()))
        d["device_error"] = rc
        return d


def random_job(rng: np.random.Generator, seed: int):
    """One job of the benchmark mix: (descriptor, sweeps)."""
    u = rng.random()
    jitter = 1.0 + rng.uniform(-0.02, 0.02)
    if u < 0.5:
        if rng.random() < 0.5:
            L = 2 * int(rng.integers(16, 513))
            shape, key = (L, L), ("ising", 2)
        else:
            L = 2 * int(rng.integers(8, 129))
            shape, key = (L, L, L), ("ising", 3)
        desc = make_desc(ISING, 2, shape, METROPOLIS, beta=BETA_C[key] * jitter, seed=seed, rng=RNG_KEYED)
    elif u < 0.8:
        q = 3 if rng.random() < 0.5 else 4
        L = 2 * int(rng.integers(8, 65))
        desc = make_desc(POTTS, q, (L, L, L), HEATBATH, beta=BETA_C[("potts", q)] * jitter, seed=seed, rng=RNG_KEYED)
    else:
        L = 2 * int(rng.integers(4, 13))
        desc = make_desc(GAUGE, 2, (L, L, L, L), HEATBATH, beta=BETA_C[("gauge", 4)] * jitter, seed=seed,
                         rng=RNG_KEYED)
    sweeps = int(rng.integers(100, 5001))
    return desc, sweeps


def run_poisson(gpu: Gpu, rate: float, n_jobs: int, seed: int = 0, sweeps_scale: float = 1.0,
                max_slots: int = 64, tick_ms: float = 10.0) -> dict:
    """Submit n_jobs with exponential inter-arrival times at `rate` jobs/s,
    wait for all of them, return latency percentiles and throughput."""
    rng = np.random.default_rng(seed)
    srv = Server(gpu, 0, max_slots, tick_ms)
    jobs = []
    t0 = time.perf_counter()
    t_next = t0
    for i in range(n_jobs):
        desc, sweeps = random_job(rng, seed * 100000 + i)
        sweeps = max(1, int(sweeps * sweeps_scale))
        t_next += rng.exponential(1.0 / rate)
        delay = t_next - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        jobs.append(srv.submit(desc, None, sweeps))
    for j in jobs:
        srv.wait(j)
    wall = time.perf_counter() - t0
    lat = np.array([srv.result(j)[2]["latency_ms"] for j in jobs])
    st = srv.stats()
    srv.close()
    return {"rate_jobs_per_s": rate, "jobs": n_jobs, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "site_updates_per_ns_busy": st["site_updates_per_ns"], "ticks": int(st["ticks"]), "wall_s": wall,
            "sweeps_scale": sweeps_scale}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="10,100,1000")
    ap.add_argument("--jobs", type=int, default=100)
    ap.add_argument("--sweeps-scale", type=float, default=1.0)
    args = ap.parse_args()
    gpu = Gpu.new()
    for r in [float(x) for x in args.rates.split(",")]:
        print(json.dumps(run_poisson(gpu, r, args.jobs, seed=int(r), sweeps_scale=args.sweeps_scale)), flush=True)


if __name__ == "__main__":
    main()
