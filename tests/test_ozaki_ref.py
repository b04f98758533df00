"""CPU tests of the Ozaki scheme II restatement (oracle/ozaki_ref.py):
exactness of the CRT reconstruction and the accuracy levels that calibrate
the device-side modulus-count estimate."""
import math

import numpy as np
import pytest

import oracle
from oracle import ozaki_ref


def test_crt_constants():
    for n in range(6, 21):
        ms, M, w, Q = ozaki_ref.crt(n)
        for a in range(len(ms)):
            for b in range(a + 1, len(ms)):
                assert math.gcd(ms[a], ms[b]) == 1
        for m, wl in zip(ms, w):
            assert wl % m == 1 and all(wl % m2 == 0 for m2 in ms if m2 != m)
        assert 4 * 2 ** (2 * Q) <= M


def test_reconstruction_is_exact():
    A = oracle.spread((6, 300), 11, 1.0)
    B = oracle.spread((300, 5), 12, 1.0)
    for n in (8, 12, 15):
        ozaki_ref.emulate(A, B, n, verify=True)


def _normerr(C, A, B):
    M, K = A.shape
    N = B.shape[1]
    ii, jj = np.indices((M, N))
    ii, jj = ii.ravel(), jj.ravel()
    val, bound = oracle.dd_entries("N", "N", M, N, K, 1.0, np.asfortranarray(A), M,
                                   np.asfortranarray(B), K, 0.0, None, M, ii, jj)
    return float(np.max(np.abs(C[ii, jj] - val) / bound)) / 2.0 ** -53


@pytest.mark.parametrize("phi,n", [(0.0, 15), (1.0, 16)])
def test_calibrated_modulus_counts_beat_native(phi, n):
    # the modulus counts the device estimate picks for these spreads are at
    # least as accurate as a plain FP64 dot product on the same inputs
    A = oracle.spread((12, 2048), 5, phi)
    B = oracle.spread((2048, 10), 6, phi)
    C, _ = ozaki_ref.emulate(A, B, n)
    assert _normerr(C, A, B) <= _normerr(A @ B, A, B) + 1e-3


@pytest.mark.parametrize("n", range(6, ozaki_ref.FP_CRT_MAX + 1))
def test_fp64_limb_crt_rounds_correctly(n):
    # the device's reconstruction, restated, against exact rounding of the
    # CRT value: random magnitudes and values next to rounding midpoints
    # (ties included), both signs and zero
    import random
    tables = ozaki_ref.fp_limb_tables(n)
    ms, M = tables[0], tables[1]
    rng = random.Random(n)
    xs = [0, 1, -1, M // 4 - 1, -(M // 4 - 1)]
    top = M.bit_length() - 3
    for _ in range(1500):
        bits = rng.randint(1, top)
        x = rng.getrandbits(bits)
        if x.bit_length() > 60 and rng.random() < 0.5:  # a midpoint of two doubles, or one away
            s = x.bit_length() - 53
            x = ((x >> s) << s) + (1 << (s - 1)) + rng.choice((-1, 0, 1))
        xs.append(x if rng.random() < 0.5 else -x)
    for x in xs:
        assert abs(x) < M // 4
        got = ozaki_ref.crt_fp64([x % m for m in ms], tables)
        assert got == float(x) and (x != 0 or math.copysign(1.0, got) > 0), (n, x, got)


def test_byte_dot_residues_match_symmetric_residues():
    # the device's residue formula, restated, against the symmetric residue
    # by definition, for every modulus, at the range ends and at random
    import random
    rng = random.Random(3)
    vs = [0, 1, -1, (1 << 62) - 1, -(1 << 62), (1 << 53) + 1, -(1 << 40)]
    vs += [rng.randrange(-(1 << 62), 1 << 62) for _ in range(3000)]
    for m in ozaki_ref.MODULI:
        for v in vs:
            r = ozaki_ref.residue_bytes(v, m)
            if m == 256:
                assert r % 256 == v % 256 and -128 <= r <= 127
            else:
                h = (m - 1) // 2
                assert r == (v + h) % m - h, (m, v)
