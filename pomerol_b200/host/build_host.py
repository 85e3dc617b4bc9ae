"""Build the drop-in host layer: lib/libpomerol_b200.so (C++ classes in
namespace Pomerol, linked against libpgx.so) and the Python extension
pomerol_b200/_pomerol (pybind11)."""
from __future__ import annotations

import subprocess
import sys
import sysconfig
from pathlib import Path

HOST = Path(__file__).resolve().parent
PKG = HOST.parent
ROOT = PKG.parent
LIB = PKG / "lib"
CXX = "g++"
FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-parameter"]
SOURCES = ["src/presets.cpp", "src/ed.cpp", "src/correlators.cpp"]


def _run(cmd):
    print(" ".join(map(str, cmd)), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def _stale(out, deps):
    return not out.exists() or any(Path(d).stat().st_mtime > out.stat().st_mtime for d in deps)


def main():
    import pybind11
    inc = ["-I", HOST / "include", "-I", ROOT / "include", "-I", "/usr/local/cuda/include"]
    headers = list((HOST / "include").rglob("*.hpp")) + [ROOT / "include/pgx.h"]
    core = LIB / "libpomerol_b200.so"
    srcs = [HOST / s for s in SOURCES]
    if _stale(core, srcs + headers + [LIB / "libpgx.so"]):
        _run([CXX, *FLAGS, "-shared", *inc, *srcs, "-L", LIB, "-lpgx", "-Wl,-rpath,$ORIGIN", "-o", core])
    ext = PKG / ("_pomerol" + sysconfig.get_config_var("EXT_SUFFIX"))
    bsrc = HOST / "bindings.cpp"
    if _stale(ext, [bsrc, core] + headers):
        py_inc = sysconfig.get_paths()["include"]
        _run([CXX, *FLAGS, "-shared", *inc, "-I", pybind11.get_include(), "-I", py_inc, bsrc, "-L", LIB,
              "-lpomerol_b200", "-lpgx", "-Wl,-rpath,$ORIGIN/lib", "-o", ext])


if __name__ == "__main__":
    main()
