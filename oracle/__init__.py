"""CPU oracle for the G2 / G / chi path (TEST INFRASTRUCTURE ONLY).

A restatement of pomerol's algorithm for this path, used by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
The product (pomerol_b200) never imports, links or executes anything here.

Parity pinning: the oracle is checked against every golden vector and
closed-form answer in the reference's tests for this path (GF1site, GF2site,
GF4site, Anderson, AndersonComplex, Susceptibility, Hamiltonian, Vertex4,
Anderson2PGF); see tests/test_oracle_golden.py.
"""
