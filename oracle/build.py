"""Build the C++ part of the CPU oracle (test infrastructure only):
oracle/_build/libg2oracle.so from oracle/g2_oracle.cpp."""
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build" / "libg2oracle.so"


def main():
    src = HERE / "g2_oracle.cpp"
    OUT.parent.mkdir(exist_ok=True)
    if OUT.exists() and OUT.stat().st_mtime > src.stat().st_mtime:
        return OUT
    cmd = ["g++", "-O3", "-march=x86-64-v2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", str(src), "-o", str(OUT)]
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    main()
