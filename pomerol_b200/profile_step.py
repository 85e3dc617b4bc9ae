"""Run the G2 step of a workload a few times on one libpgx context (for
ncu captures and stage timing): eigensolve, weights, rotation, G2; with
--chi3 N the three-point susceptibility chi3_PH(u0, u0, d0, d0) on the
N x N fermionic square instead of G2; with --batch M the first M models of
the batch workload (G on 1024 and chi_dd on 32 frequencies per model).

    python -m pomerol_b200.profile_step [--config a5] [--steps 2] [--chi3 32] [--batch 64]
"""
import argparse
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="a5")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--kernels", action="store_true", help="per-kernel event times of the last step")
    ap.add_argument("--chi3", type=int, default=0, help="chi3 on an N x N square instead of G2")
    ap.add_argument("--batch", type=int, default=0, help="the first M models of the batch workload")
    a = ap.parse_args()
    import torch  # noqa: F401  (CUDA context for the process)
    from .workloads import BatchRun, Chi3Run, EngineRun, Problem, b64_params, matsubara_cube, matsubara_square
    if a.batch:
        run = BatchRun(b64_params()[:a.batch])
        for s in range(a.steps):
            last = a.kernels and s == a.steps - 1
            if last:
                run.eng.profile_begin()
            run.eng.timer_begin()
            t0 = time.perf_counter()
            G, X = run.step()
            ms = run.eng.timer_end()
            if last:
                for k in run.eng.profile_end():
                    print(f"  {k['name']:44s} x{k['launches']:<4d} {k['ms']:9.3f} ms  "
                          f"{k['flops'] / max(k['ms'], 1e-9) / 1e9:9.3f} TFLOP/s")
            print(f"step {s}: device {ms:.1f} ms, wall {1e3 * (time.perf_counter() - t0):.1f} ms, "
                  f"blocks {len(run.dims)}, G terms {run.nterms_G:.3e}, chi terms {run.nterms_X:.3e}", flush=True)
        return
    prob = Problem(a.config)
    if a.chi3:
        _, z = matsubara_square(prob.beta, a.chi3)
        run = Chi3Run(prob)
    else:
        _, z = matsubara_cube(prob.beta, prob.nfreq)
        run = EngineRun(prob)
    for s in range(a.steps):
        t0 = time.perf_counter()
        last = a.kernels and s == a.steps - 1
        if last:
            run.eng.profile_begin()
        run.eng.timer_begin()
        v = run.step(z)
        ms = run.eng.timer_end()
        if last:
            for k in run.eng.profile_end():
                print(f"  {k['name']:40s} x{k['launches']:<3d} {k['ms']:9.3f} ms  "
                      f"{k['flops'] / max(k['ms'], 1e-9) / 1e9:9.3f} TFLOP/s  {k['bytes'] / max(k['ms'], 1e-9) / 1e6:9.2f} GB/s")
        extra = "" if a.chi3 else f"g2 {run.eng.g2_timing()}, "
        print(f"step {s}: device {ms:.1f} ms, wall {1e3 * (time.perf_counter() - t0):.1f} ms, "
              f"{extra}|v|max {np.abs(v).max():.4e}", flush=True)


if __name__ == "__main__":
    main()
