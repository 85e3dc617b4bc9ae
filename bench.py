"""Benchmark of the G2 path on B200: full two-particle Green's function
(block eigensolve + operator rotation + Lehmann sum) of the Anderson 1+5
impurity (dim 4096, chi_(u0,d0,u0,d0) on the 16^3 fermionic cube, beta=20).

Metric: G2 Lehmann term*freq evaluations per second = N_quad * N_freq / step
time, where N_quad counts the state quadruples the reference enumerates
(all four rotated elements non-zero, w1+w2+w3+w4 > 1e-16) and N_freq the
frequency triples.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Our arm, per step (value): eigensolve, weights, rotation of c^+/c and the G2
sum on one libpgx context with the block Hamiltonians resident in HBM.  e2e:
the same through the drop-in API from the Hamiltonian expression, with every
host<->device copy inside the timed region.  Multi-GPU: one process per GPU,
each rank computes its own frequency slab (weak scaling, no collective in the
data path), time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIG = "a5"
NZ_TOL = 1e-12
COEF_TOL = 1e-16


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default=CONFIG)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(2)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def flush_l2(buf):
    if buf is not None:
        buf.add_(1.0)


def fp64_peak_tflops(torch):
    """Measured FP64 reference: cuBLAS DGEMM 8192^3 via torch.matmul (best of 3)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


# ------------------------------------------------------------------ CPU side
def cpu_sample(config, seconds_target=12.0, nthreads=0):
    """The reference's algorithm (oracle/g2_oracle.cpp restatement: chase
    enumeration, TermList merging, OpenMP frequency loop) on a bounded sample
    of the workload: rows of index1 of the largest block chain, all triples.
    Returns (rate term*freq/s, seconds, description, threads)."""
    from oracle import ed as EDm
    from oracle import g2c
    from oracle import lehmann as L
    from oracle import model as M
    from pomerol_b200.workloads import CONFIGS, a5_params, matsubara_cube

    cfg = CONFIGS[config]
    if config == "a5":
        U, epsd, eps, V, beta = a5_params(0)
        mdl = M.make_model(M.anderson(U, epsd, eps, V))
        site = "C"
    elif config == "plaquette":
        mdl, beta, site = M.make_model(M.plaquette()), cfg["beta"], "A"
    else:
        raise ValueError(config)
    ed = EDm.ED(mdl, beta)
    u, d = mdl.info.getIndex(site, 0, 1), mdl.info.getIndex(site, 0, 0)
    parts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
    sizes = [np.prod([len(mdl.blocks[b]) for b in p["b"]]) for p in parts]
    k = int(np.argmax(sizes))
    _, z = matsubara_cube(beta, cfg["nfreq"])
    d1 = len(mdl.blocks[parts[k]["b"][0]])
    threads = nthreads or g2c.lib().g2o_max_threads()
    # index1 rows strided across the whole block (eigenvalues ascend, so the
    # hot low-energy rows and the cold ones are both represented)
    nrows = 2
    while True:
        step = max(1, d1 // nrows)
        t0 = time.perf_counter()
        _, nq, terms = g2c.evaluate(ed, parts, z, rows=(k, 0, d1, step), nthreads=threads)
        dt = time.perf_counter() - t0
        if dt > seconds_target / 3 or step == 1:
            break
        nrows = min(d1, max(nrows + 1, int(nrows * min(8.0, seconds_target / 3 / max(dt, 1e-3)))))
    rate = nq * len(z) / dt
    desc = (f"reference algorithm restated (oracle/g2_oracle.cpp): block chain {k} of {len(parts)} "
            f"(blocks {[len(mdl.blocks[b]) for b in parts[k]['b']]}), every {step}-th index1 row of {d1}, "
            f"{nq} quadruples, {int(terms.sum())} merged terms, {len(z)} triples, {dt:.2f} s on {threads} threads")
    return rate, dt, desc, threads, (k, step)


def run_reference(args, rank, world):
    unit = "term*freq/s"
    if rank != 0:
        return
    try:
        from oracle import g2c
        g2c.lib()
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"oracle build failed: {e}"}))
        return
    rate, dt, desc, threads, (k, step) = cpu_sample(args.config, seconds_target=8.0)
    times, rates = [], []
    for i in range(args.warmup + args.steps):
        r, t, _, _, _ = cpu_sample_fixed(args.config, k, step, threads)
        if i >= args.warmup:
            rates.append(r)
        if i >= args.warmup:
            times.append(t)
    ms = 1e3 * float(np.mean(times))
    value = float(np.mean(rates))
    line = {"metric": "G2 Lehmann term*freq evals/s", "value": value, "unit": unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "anderson_1+5_dim4096_chi_u0d0u0d0_16cube_beta20", "sample": desc},
            "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


_CPU_CACHE = {}


def cpu_sample_fixed(config, k, step, threads):
    from oracle import ed as EDm
    from oracle import g2c
    from oracle import lehmann as L
    from oracle import model as M
    from pomerol_b200.workloads import CONFIGS, a5_params, matsubara_cube
    if config not in _CPU_CACHE:
        cfg = CONFIGS[config]
        if config == "a5":
            U, epsd, eps, V, beta = a5_params(0)
            mdl, site = M.make_model(M.anderson(U, epsd, eps, V)), "C"
        else:
            mdl, beta, site = M.make_model(M.plaquette()), cfg["beta"], "A"
        ed = EDm.ED(mdl, beta)
        u, d = mdl.info.getIndex(site, 0, 1), mdl.info.getIndex(site, 0, 0)
        parts = L.g2_parts(ed, ed.c(u), ed.c(d), ed.cdag(u), ed.cdag(d))
        _, z = matsubara_cube(beta, cfg["nfreq"])
        _CPU_CACHE[config] = (ed, parts, z)
    ed, parts, z = _CPU_CACHE[config]
    t0 = time.perf_counter()
    d1 = len(ed.E[parts[k]["b"][0]])
    _, nq, _ = g2c.evaluate(ed, parts, z, rows=(k, 0, d1, step), nthreads=threads)
    dt = time.perf_counter() - t0
    return nq * len(z) / dt, dt, None, threads, None


# ------------------------------------------------------------------ GPU side
def run_ours(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    from pomerol_b200 import pgx
    from pomerol_b200.workloads import EngineRun, Problem, matsubara_cube

    prob = Problem(args.config, device=local_rank)
    # weak scaling: rank r owns the slab shifted by r * nfreq along n1
    idx, z = matsubara_cube(prob.beta, prob.nfreq)
    z = z.copy()
    z[:, 0] += 1j * 2 * np.pi * rank * prob.nfreq / prob.beta
    run = EngineRun(prob, device=local_rank)
    run.step(z)
    nquad = run.eng.g2_count(run.parts, COEF_TOL, NZ_TOL)
    nfreq = len(z)
    l2buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    # per-kernel CUDA-event ranges stay on through warm-up (their events are
    # created there) and the timed steps; the timed steps' stats give the roofline
    run.eng.profile_begin()
    for _ in range(args.warmup):
        run.step(z)
    run.eng.profile_end()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    times = []
    launches0 = pgx.launch_count()
    run.eng.profile_begin()
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            flush_l2(l2buf)
            torch.cuda.synchronize()
            run.eng.timer_begin()
            out = run.step(z)
            times.append(run.eng.timer_end())
    launches = pgx.launch_count() - launches0
    kstats = run.eng.profile_end()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms = float(np.mean(times))
    t_max = ms
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        t_max = float(t.item())
    units = float(nquad) * nfreq * world
    value = units / (t_max / 1e3)

    # e2e through the drop-in API from the Hamiltonian expression
    e2e_times = []
    triples = [tuple(x) for x in z]  # the caller's input, in host memory before the timed region
    # untimed calls first: the drop-in objects of one call live until the next
    # call replaces them, so the first two calls each set up a GPU context
    e2e_warm = max(2, args.warmup)
    for i in range(max(2, args.steps // 2) + e2e_warm):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        v = prob.run_api(triples)
        torch.cuda.synchronize()
        if i >= e2e_warm:
            e2e_times.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(e2e_times))
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    agree = float(np.abs(v - out).max() / max(np.abs(out).max(), 1e-300))

    if rank != 0:
        return
    # dominant kernel of the timed steps: algorithmic FLOPs per launch over its
    # average event-timed duration, against the measured FP64 GEMM peak
    top = kstats[0] if kstats else None
    peak = fp64_peak_tflops(torch)
    achieved = None
    if top and top["ms"] > 0 and top["flops"] > 0:
        achieved = (top["flops"] / top["launches"]) / (top["ms"] / top["launches"] / 1e3) / 1e12
    traffic = None
    tf = ROOT / "profiles" / "roofline_traffic.json"
    if tf.exists() and top:
        try:
            traffic = json.loads(tf.read_text()).get(args.config, {}).get(top["name"])
        except Exception:
            traffic = None
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            rate, dt, desc, threads, _ = cpu_sample(args.config)
            cpu = {"value": rate, "unit": "term*freq/s", "cores": threads, "kind": "port", "sample": desc}
        except Exception as e:
            cpu = {"value": None, "unit": "term*freq/s", "cores": None, "kind": "port", "sample": f"failed: {e}"}
    line = {
        "metric": "G2 Lehmann term*freq evals/s", "value": value, "unit": "term*freq/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "anderson_1+5_dim4096_chi_u0d0u0d0_16cube_beta20", "n_quad": nquad,
                   "n_freq_per_rank": nfreq, "blocks": len(prob.dims), "max_block": max(prob.dims),
                   "g2_parts": len(run.parts), "l2": "flushed (256 MB write) between timed steps; working set > L2",
                   "stages_in_step": "eigh+weights+rotate(c+,c)+G2", "pole_resolution": 1e-8},
        "gpu_launches": launches // max(1, args.steps) * args.steps,
        "clocks": clk.summary(),
        "e2e": {"value": float(nquad) * nfreq * world / e2e_s, "unit": "term*freq/s",
                "h2d_bytes_per_step": int(run.h2d_bytes + z.nbytes),
                "d2h_bytes_per_step": int(out.nbytes), "seconds_per_step": e2e_s,
                "path": "drop-in API (Hamiltonian..TwoParticleGFContainer.computeAll) from the expression",
                "max_rel_diff_vs_value_leg": agree},
        "roofline": {"kernel": top["name"] if top else None,
                     "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": (achieved / peak) if (achieved and peak) else None, "traffic": traffic,
                     "peak_source": "measured live: cuBLAS FP64 DGEMM 8192^3 (torch.matmul float64); "
                                    "MEASURED_PEAKS.json has no FP64 figure (FP64 arithmetic, CUDA-core FMA pipe)",
                     "launches_per_step": (top["launches"] / args.steps) if top else None,
                     "ms_per_launch": (top["ms"] / top["launches"]) if top else None,
                     "flops_per_launch": (top["flops"] / top["launches"]) if top else None,
                     "kernels_ms_per_step": {k["name"]: round(k["ms"] / args.steps, 4) for k in kstats}},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
