"""Run the G2 step of a workload a few times on one libpgx context (for
ncu captures and stage timing): eigensolve, weights, rotation, G2.

    python -m pomerol_b200.profile_step [--config a5] [--steps 2]
"""
import argparse
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="a5")
    ap.add_argument("--steps", type=int, default=2)
    a = ap.parse_args()
    import torch  # noqa: F401  (CUDA context for the process)
    from .workloads import EngineRun, Problem, matsubara_cube
    prob = Problem(a.config)
    _, z = matsubara_cube(prob.beta, prob.nfreq)
    run = EngineRun(prob)
    for s in range(a.steps):
        t0 = time.perf_counter()
        run.eng.timer_begin()
        v = run.step(z)
        ms = run.eng.timer_end()
        print(f"step {s}: device {ms:.1f} ms, wall {1e3 * (time.perf_counter() - t0):.1f} ms, "
              f"g2 {run.eng.g2_timing()}, |v|max {np.abs(v).max():.4e}", flush=True)


if __name__ == "__main__":
    main()
