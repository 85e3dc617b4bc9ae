"""Extract the reference's numeric golden vectors into reference_kats.json.

The values are read as text from the reference's Catch2 test sources (they
are literal arrays there); the model parameters that go with them are
written below next to the file:line they come from.  Run from the repository
root with the reference checkout at REF (default /root/reference):

    python tests/golden/make_golden.py [REF]
"""
import json
import re
import sys
from pathlib import Path

REF = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
OUT = Path(__file__).with_name("reference_kats.json")

NUM = r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?"


def block_after(text, marker, occurrence=0):
    i = -1
    for _ in range(occurrence + 1):
        i = text.index(marker, i + 1)
    j = text.index(";", i)
    # drop // comments line by line before the entries are split
    return "\n".join(line.split("//")[0] for line in text[i:j].splitlines())


def complex_list(block):
    """Parse 'a - b * I,' / 'c * I' style entries of an Eigen << list."""
    body = block.split("<<", 1)[1]
    out = []
    for ent in body.split(","):
        ent = ent.split("//")[0].strip()
        if not ent:
            continue
        m = re.fullmatch(rf"({NUM})\s*([-+])\s*({NUM})\s*\*\s*I", ent)
        if m:
            im = float(m.group(3)) * (1 if m.group(2) == "+" else -1)
            out.append([float(m.group(1)), im])
            continue
        m = re.fullmatch(rf"({NUM})\s*\*\s*I", ent)
        if m:
            out.append([0.0, float(m.group(1))])
            continue
        out.append([float(ent), 0.0])
    return out


def real_list(block):
    body = block.split("<<", 1)[1]
    return [float(x.split("//")[0]) for x in body.split(",") if x.split("//")[0].strip()]


def main():
    t = (REF / "test/Anderson2PGFTest.cpp").read_text()
    a2 = real_list(block_after(t, "chi_ref <<"))
    t = (REF / "test/GF4siteTest.cpp").read_text()
    g4 = complex_list(block_after(t, "G_ref <<"))
    t = (REF / "test/GF2siteTest.cpp").read_text()
    g2 = complex_list(block_after(t, "G_ref <<"))
    t = (REF / "test/AndersonTest.cpp").read_text()
    au = complex_list(block_after(t, "G_ref_up <<"))
    ad = complex_list(block_after(t, "G_ref_down <<"))
    t = (REF / "test/HamiltonianTest.cpp").read_text()
    e0 = float(re.search(rf"E_ref = ({NUM})", t).group(1))
    t = (REF / "test/3PSusc3siteTest.cpp").read_text()
    chi3 = [complex_list(block_after(t, "chi3_ref <<", q)) for q in range(3)]
    kats = {
        "anderson2pgf": {
            "source": "test/Anderson2PGFTest.cpp:37-58,97-126",
            "U": 0.5, "mu": 0.25, "beta": 26.0,
            "levels": [1.02036910873357, -1.02036910873357],
            "hoppings": [0.296439333614347, 0.296439333614347],
            "pole_resolution": 1e-5, "coefficient_tolerance": 1e-8,
            "freqs": "z = (i*pi/beta + i*2pi/beta, i*(2k+1)*pi/beta, i*pi/beta), k=0..9",
            "chi_uuuu": a2, "tol": 1e-6,
        },
        "gf4site": {
            "source": "test/GF4siteTest.cpp:36-62,102-108",
            "beta": 10.0,
            "coulomb": [["A", 1.0, -0.5], ["B", 2.0, -1.1], ["C", 3.0, -0.7], ["D", 4.0, -1.1]],
            "hopping": [["A", "B", -1.3], ["B", "C", -0.45], ["C", "D", -0.127], ["A", "D", -0.255]],
            "G_A_down": g4, "tol": 1e-6,
        },
        "gf2site": {
            "source": "test/GF2siteTest.cpp:34-121",
            "U": 1.0, "mu": 0.5, "beta": 10.0, "t": -1.0,
            "G_A_down": g2, "tol": 1e-8,
        },
        "anderson": {
            "source": "test/AndersonTest.cpp:31-124",
            "U": 3.7, "mu_over_U": 0.6, "h": 0.1, "V": 1.0, "epsilon": 2.3, "beta": 20.0,
            "G_up": au, "G_down": ad, "tol": 1e-8,
        },
        "chi3_3site": {
            "source": "test/3PSusc3siteTest.cpp:24-157",
            "U": 4.0, "mu": 2.4, "t": 1.0, "beta": 5.0,
            "sites": ["A", "B", "C"],
            "n": [-1, 0, 1],
            "PP": {"ops": [["A", "up"], ["C", "up"], ["A", "down"], ["C", "down"]], "chi3": chi3[0]},
            "PH": {"ops": [["A", "up"], ["A", "up"], ["C", "down"], ["C", "down"]], "chi3": chi3[1]},
            "xPH": {"ops": [["A", "up"], ["C", "up"], ["C", "down"], ["A", "down"]], "chi3": chi3[2]},
            "layout": "chi3[(n1 + 1) * 3 + (n2 + 1)] for n1, n2 in n",
            "tol": 1e-10,
        },
        "hamiltonian": {
            "source": "test/HamiltonianTest.cpp:31-75",
            "E0": e0, "tol": 1e-7,
        },
    }
    OUT.write_text(json.dumps(kats, indent=1) + "\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
