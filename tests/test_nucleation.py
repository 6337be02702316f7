"""Nucleation Monte Carlo on the GPU (gw_fopt_b200/csrc/nucleation.cu) against its
CPU restatement (oracle/nucleation.py).

The generator is Philox4x32-10; its output is checked against the published
known-answer vectors of the algorithm (Random123 kat_vectors, philox4x32_10).
The device and the oracle take the same candidates and decisions: accepted
positions are bitwise equal and times agree to 1e-12 (the device's log/exp and
the host's differ in the last bits; the tests check that no decision lies that
close to its threshold).
"""
import numpy as np
import pytest

from oracle import nucleation as ON
from gw_fopt_b200 import many_bubbles as mb

KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]

CASES = [(40, 8.0, 11), (120, 20.0, 12345), (60, 5.0, 2 ** 33 + 7), (1, 6.0, 3), (0, 6.0, 4)]


def test_philox_known_answers():
    for ctr, key, want in KAT:
        assert ON.philox4x32(ctr, key) == want


def test_oracle_draw_is_causal_and_shaped():
    interior, exterior, att = ON.exponential_nucleation(80, 10.0, 99, max_rejections=2000)
    assert interior.shape == (80, 4) and exterior.shape == (480, 4) and att >= 1
    assert interior[0, 0] == 0.0 and np.all(np.diff(interior[:, 0]) > 0)
    mb.LatticeBubbles(mb.EmptyLattice(), interior, exterior)  # raises when not causal


@pytest.mark.gpu
def test_device_nucleation_matches_oracle(gpu_available):
    from gw_fopt_b200 import nucleation as NU
    ns = [c[0] for c in CASES]
    out = NU.exponential_nucleation(ns, [c[1] for c in CASES], [c[2] for c in CASES], max_rejections=3000)
    for (n, beta, seed), (interior, exterior) in zip(CASES, out):
        ri, re, _ = ON.exponential_nucleation(n, beta, seed, max_rejections=3000)
        assert interior.shape == ri.shape and exterior.shape == re.shape
        assert np.array_equal(interior[:, 1:], ri[:, 1:])
        assert np.array_equal(exterior[:, 1:], re[:, 1:])
        assert np.allclose(interior[:, 0], ri[:, 0], rtol=0, atol=1e-12)
        if n:
            mb.LatticeBubbles(mb.EmptyLattice(), interior, exterior)


@pytest.mark.gpu
def test_device_nucleation_rejects_bad_input(gpu_available):
    from gw_fopt_b200 import _lib as L
    from gw_fopt_b200 import nucleation as NU
    with pytest.raises(L.BgwError, match="n_bubbles"):
        NU.exponential_nucleation([-1], [5.0], [1])
    with pytest.raises(L.BgwError, match="beta"):
        NU.exponential_nucleation([10], [0.0], [1])
