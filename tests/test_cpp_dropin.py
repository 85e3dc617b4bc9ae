"""The drop-in boundary from C++: tests/cpp/dropin_g2.cpp is written as a
pomerol user would write it (namespace Pomerol, the reference's class names
and call sequence), compiled against pomerol_b200/host/include and linked
with libpomerol_b200.so.  It must compile without a GPU; on a GPU it must
reproduce the golden values of the reference's two-bath Anderson G2 test
(Anderson2PGFTest.cpp:46-58, both computeAll modes, 1e-6) read from
tests/golden/reference_kats.json."""
import json
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "dropin_g2.cpp"
LIB = ROOT / "pomerol_b200" / "lib"


def _build(out: Path):
    if not (LIB / "libpomerol_b200.so").exists():
        pytest.fail("libpomerol_b200.so is not built (python pomerol_b200/host/build_host.py)")
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", str(ROOT / "pomerol_b200" / "host" / "include"),
           "-I", str(ROOT / "include"), "-I", "/usr/local/cuda/include", str(SRC), "-L", str(LIB),
           "-lpomerol_b200", "-lpgx", f"-Wl,-rpath,{LIB}", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_dropin_program_compiles_against_the_headers(tmp_path):
    exe = _build(tmp_path / "dropin_g2")
    assert exe.exists()


@pytest.mark.gpu
def test_dropin_program_reproduces_anderson2pgf(tmp_path):
    k = json.loads((ROOT / "tests" / "golden" / "reference_kats.json").read_text())["anderson2pgf"]
    exe = _build(tmp_path / "dropin_g2")
    params = tmp_path / "params.txt"
    lines = [f"{k['U']!r} {k['mu']!r} {k['beta']!r} {k['pole_resolution']!r} {k['coefficient_tolerance']!r} "
             f"{k['tol']!r}",
             f"{len(k['levels'])} " + " ".join(f"{e!r} {t!r}" for e, t in zip(k["levels"], k["hoppings"])),
             f"{len(k['chi_uuuu'])} " + " ".join(repr(v) for v in k["chi_uuuu"])]
    params.write_text("\n".join(lines) + "\n")
    r = subprocess.run([str(exe), str(params)], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr)
    assert r.returncode == 0, r.stderr
    assert "0 mismatches of 40 values" in r.stdout
