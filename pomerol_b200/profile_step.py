"""Run the G2 step of a workload a few times on one libpgx context (for
ncu captures and stage timing): eigensolve, weights, rotation, G2; with
--chi3 N the three-point susceptibility chi3_PH(u0, u0, d0, d0) on the
N x N fermionic square instead of G2; with --batch M the first M models of
the batch workload (G on 1024 and chi_dd on 32 frequencies per model); with
--chain the drop-in chain of a workload stage by stage (Hamiltonian,
DensityMatrix, field operators, G_u0 on 256 fermionic and chi_zz on 48 bosonic
frequencies, then G2 on the N x N x N cubes given by --g2-cubes).

    python -m pomerol_b200.profile_step [--config a5] [--steps 2] [--chi3 32] [--batch 64]
    python -m pomerol_b200.profile_step --config ring8 --chain --g2-cubes 2 4
"""
import argparse
import time

import numpy as np


def _unit(name):
    """The split-product ranges record int8 operations, the others FP64 ones."""
    return "TOPS(i8)" if name.startswith("oz_gemm") else "TFLOP/s "


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="a5")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--kernels", action="store_true", help="per-kernel event times of the last step")
    ap.add_argument("--chi3", type=int, default=0, help="chi3 on an N x N square instead of G2")
    ap.add_argument("--batch", type=int, default=0, help="the first M models of the batch workload")
    ap.add_argument("--chain", action="store_true", help="time the drop-in chain stage by stage")
    ap.add_argument("--g2-cubes", type=int, nargs="*", default=[], help="cube sides for the G2 stage of --chain")
    ap.add_argument("--split", action="store_true",
                    help="anchored G2 with its stacked products on the int8 tensor cores (PGX_G2_SPLIT_I8); "
                         "with --chain each cube also runs in FP64 for the error")
    ap.add_argument("--anchor-tol", type=float, default=1e-16, help="anchor weight threshold of the G2 sum")
    ap.add_argument("--slices", type=int, default=6, help="base-254 digits per element of the split products")
    ap.add_argument("--fp64", action="store_true", help="with --split: also run the plain FP64 form (same sum)")
    ap.add_argument("--cta-pair", type=int, default=0,
                    help="split-product tiles: 0 for 128 x 256 on single CTAs (default), 1 for 256 x 256 on CTA pairs")
    ap.add_argument("--autotune", action="store_true",
                    help="measure the GEMM tile classes on one step (after one untimed step) before timing")
    a = ap.parse_args()
    if a.chain:
        chain(a.config, a.g2_cubes, a.kernels, a.split)
        return
    import torch  # noqa: F401  (CUDA context for the process)
    from .workloads import BatchRun, Chi3Run, EngineRun, Problem, b64_params, matsubara_cube, matsubara_square
    if a.batch:
        run = BatchRun(b64_params()[:a.batch])
        if a.autotune:
            autotune(run.eng, run.step)
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
        run = EngineRun(prob, split=a.split, anchor_tol=a.anchor_tol, slices=a.slices)
        run.eng.set_split_cta_pair(a.cta_pair)
    if a.autotune:
        autotune(run.eng, lambda: run.step(z))
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
                      f"{k['flops'] / max(k['ms'], 1e-9) / 1e9:9.3f} {_unit(k['name'])}  "
                      f"{k['bytes'] / max(k['ms'], 1e-9) / 1e6:9.2f} GB/s")
        extra = "" if a.chi3 else f"g2 {run.eng.g2_timing()}, "
        print(f"step {s}: device {ms:.1f} ms, wall {1e3 * (time.perf_counter() - t0):.1f} ms, "
              f"{extra}|v|max {np.abs(v).max():.4e}", flush=True)
    if a.fp64 and a.split and not a.chi3:
        from .pgx import PGX_G2_ANCHORED
        run.eng.profile_begin()
        run.eng.timer_begin()
        v64 = run.g2(run.parts, z, flags=PGX_G2_ANCHORED)
        ms = run.eng.timer_end()
        for k in run.eng.profile_end()[:6]:
            print(f"  {k['name']:40s} x{k['launches']:<3d} {k['ms']:9.3f} ms  "
                  f"{k['flops'] / max(k['ms'], 1e-9) / 1e9:9.3f} TFLOP/s", flush=True)
        print(f"plain FP64 form (G2 only, same anchored sum): device {ms:.1f} ms; split vs FP64: max|diff| / max|G2| "
              f"{np.abs(v - v64).max() / np.abs(v64).max():.2e}", flush=True)


def autotune(eng, step):
    step()  # sizes every buffer
    eng.autotune_begin()
    step()
    t0 = time.perf_counter()
    n = eng.autotune_end()
    print(f"autotune: {n} size buckets off the padding rule ({1e3 * (time.perf_counter() - t0):.1f} ms)", flush=True)


def chain(config, cubes, kernels=False, split=False):
    import torch  # noqa: F401  (CUDA context for the process)
    from . import _pomerol as P
    from .workloads import EngineRun, Problem, matsubara_cube
    prob = Problem(config)
    t = time.perf_counter()
    H = P.Hamiltonian(prob.S)
    H.prepare(prob.HExpr, prob.hs)
    H.compute()
    t1 = time.perf_counter()
    print(f"Hamiltonian prepare + compute: {t1 - t:.2f} s ({len(prob.dims)} blocks, largest {max(prob.dims)})")
    rho = P.DensityMatrix(prob.S, H, prob.beta)
    rho.prepare()
    rho.compute()
    if prob.dm_trunc:
        rho.truncateBlocks(prob.dm_trunc)
    ops = P.FieldOperatorContainer(prob.ii, prob.hs, prob.S, H, {prob.u0, prob.d0})
    ops.prepareAll(prob.hs)
    ops.computeAll()
    t2 = time.perf_counter()
    print(f"DensityMatrix + rotation of c+, c (u0, d0): {t2 - t1:.3f} s")
    G = P.GreensFunction(prob.S, H, ops.getAnnihilationOperator(prob.u0), ops.getCreationOperator(prob.u0), rho)
    G.prepare()
    G.compute()
    g = G.values([1j * np.pi * (2 * n + 1) / prob.beta for n in range(256)])
    t3 = time.perf_counter()
    print(f"G_u0 on 256 fermionic frequencies: {t3 - t2:.3f} s, G(0) = {g[0]:.10e}")
    chi = {}
    for x in (prob.u0, prob.d0):
        for y in (prob.u0, prob.d0):
            nx = P.QuadraticOperator(prob.ii, prob.hs, prob.S, H, x, x)
            ny = P.QuadraticOperator(prob.ii, prob.hs, prob.S, H, y, y)
            for n in (nx, ny):
                n.prepare(prob.hs)
                n.compute()
            c = P.Susceptibility(prob.S, H, nx, ny, rho)
            c.prepare()
            c.compute()
            chi[(x, y)] = np.array(c.values([2j * np.pi * m / prob.beta for m in range(48)]))
    u, d = prob.u0, prob.d0
    zz = 0.25 * (chi[(u, u)] - chi[(u, d)] - chi[(d, u)] + chi[(d, d)])
    t4 = time.perf_counter()
    print(f"chi_zz on 48 bosonic frequencies (4 pair susceptibilities): {t4 - t3:.3f} s, chi_zz(0) = {zz[0]:.10e}")
    if cubes:
        runs = [("fp64", EngineRun(prob))] + ([("split-i8", EngineRun(prob, split=True))] if split else [])
        for i, n in enumerate(cubes):
            _, z = matsubara_cube(prob.beta, n)
            ref = None
            for label, run in runs:
                prof = kernels and i == len(cubes) - 1
                if prof:
                    run.eng.profile_begin()
                run.eng.timer_begin()
                t = time.perf_counter()
                v = run.step(z)
                ms = run.eng.timer_end()
                extra = ""
                if ref is None:
                    ref = v
                else:
                    extra = f", max|diff| / max|G2| vs fp64 {np.abs(v - ref).max() / np.abs(ref).max():.2e}"
                print(f"G2 step [{label}] (eigensolve + weights + rotation + G2) on {len(z)} triples: device {ms:.0f} "
                      f"ms, wall {time.perf_counter() - t:.1f} s, g2 {run.eng.g2_timing()['total_ms'] / 1e3:.1f} s"
                      f"{extra}", flush=True)
                if prof:
                    for k in run.eng.profile_end()[:10]:
                        print(f"  {k['name']:48s} x{k['launches']:<5d} {k['ms'] / 1e3:8.2f} s  "
                              f"{k['flops'] / max(k['ms'], 1e-9) / 1e9:7.2f} TFLOP/s", flush=True)


if __name__ == "__main__":
    main()
