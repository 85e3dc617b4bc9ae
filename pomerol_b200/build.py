"""Build the in-tree native libraries for B200 (sm_100a).

    python -m pomerol_b200.build          # libpgx.so (CUDA engine + C ABI)

Outputs go to pomerol_b200/lib/.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CU_SOURCES = ["pgx_api.cu", "pgx_eigh.cu", "pgx_lehmann.cu", "pgx_g2.cu", "pgx_g2a.cu", "pgx_noalloc.cu", "pgx_assemble.cu", "pgx_vjp.cu", "pgx_chi3.cu", "pgx_tune.cu",
              "pgx_ozaki.cu"]


def _run(cmd):
    print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_pgx(verbose_ptxas: bool = False) -> Path:
    LIB.mkdir(exist_ok=True)
    out = LIB / "libpgx.so"
    deps = [CSRC / s for s in CU_SOURCES] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include/pgx.h"]
    if not _stale(out, deps):
        return out
    objs, cmds = [], []
    for s in CU_SOURCES:
        o = LIB / (Path(s).stem + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", ROOT / "include",
               "-c", CSRC / s, "-o", o]
        if verbose_ptxas:
            cmd[1:1] = ["-Xptxas", "-v"]
        cmds.append(cmd)
        objs.append(o)
    # translation units compile independently: one nvcc per core
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(_run, cmds))
    _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-lcudart"])
    for o in objs:
        o.unlink()
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    build_pgx(verbose_ptxas="-v" in argv)


if __name__ == "__main__":
    main()
