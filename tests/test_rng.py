"""Random-number pins (CPU).

* std::mt19937 seeding of the JKISS slots (GGEMSPseudoRandomGenerator.cc:140-167):
  the C++ standard's 10000th-output check, the product's seeding against
  numpy's MT19937, and the per-device skip.
* KissUniform's double division (GGEMSKissEngine.hh:72-74) replaced by one
  double multiply, and that by one single-precision fused multiply-add (the
  GPU's form): both checked over every float value a uint32 sum can round to
  (83,886,080 values).
* JKISS sequence: the oracle's and the product's state after N draws.
"""

import ctypes as C

import numpy as np

import scenes
from ggems_b200 import abi


def _lib():
    from ggems_b200._native import lib
    return lib


def test_mt19937_standard_pin():
    from numpy.random import MT19937
    bg = MT19937(0)
    bg._legacy_seeding(5489)
    assert int(bg.random_raw(10000)[-1]) == 4123659995  # [rand.predef] of the C++ standard


def test_product_seeding_matches_mt19937():
    lib = _lib()
    st = np.zeros(5 * abi.GG_MAXIMUM_PARTICLES, np.uint32)
    assert lib.gg_seed_random_states(abi.ptr(st, C.c_uint32), abi.GG_MAXIMUM_PARTICLES, 777, 0) == 0
    ref = scenes.seed_states(777)
    assert np.array_equal(st.reshape(5, -1), ref)
    # second device: the next 4 * MAXIMUM_PARTICLES outputs
    st2 = np.zeros(5 * abi.GG_MAXIMUM_PARTICLES, np.uint32)
    assert lib.gg_seed_random_states(abi.ptr(st2, C.c_uint32), 1000, 777, abi.GG_MAXIMUM_PARTICLES) == 0
    ref2 = scenes.seed_states(777, slots=1000, skip=abi.GG_MAXIMUM_PARTICLES)
    assert np.array_equal(st2.reshape(5, -1)[:, :1000], ref2[:, :1000])
    assert not st2[4 * abi.GG_MAXIMUM_PARTICLES:].any()


def _float_values_of_uint32():
    """All distinct float32 values (float)u takes for u in [0, 2^32)."""
    small = np.arange(1 << 24, dtype=np.float64)
    parts = [small]
    for e in range(24, 32):
        m = np.arange(1 << 23, 1 << 24, dtype=np.float64)
        parts.append(m * float(1 << (e - 23)))
    parts.append(np.array([4294967296.0]))
    return parts


def test_kiss_scale_is_exact():
    c = float(np.float32(1.0) - np.float32(1.0) / np.float32(1 << 23))
    scale = (1.0 / 4294967295.0) * c
    n = 0
    for x in _float_values_of_uint32():
        ref = ((x / 4294967295.0) * c).astype(np.float32)
        fast = (x * scale).astype(np.float32)
        assert np.array_equal(ref, fast)
        n += x.size
    assert n == 83886081  # includes 2^32 (the rounding of 0xffffffff)


def test_kiss_scale_single_precision_fma_is_exact():
    """The transport kernel's form: fma(x, c, x * 2^-32) in float32 with
    c = -(2^-23 - 2^-32) * 2^-32.  x * c + x * 2^-32 = (2^32 - 511) m 2^(k-64)
    for x = m 2^k (m < 2^24) needs at most 56 bits, so it is exact in x87
    extended precision (64 bits) and one cast to float32 is the fused
    multiply-add's single rounding."""
    c = float.fromhex("-0x1.ffp-56")
    assert c == -(2.0 ** -23 - 2.0 ** -32) * 2.0 ** -32 and float(np.float32(c)) == c
    assert np.finfo(np.longdouble).nmant >= 63
    k = 1.0 - 2.0 ** -23
    n = 0
    for x in _float_values_of_uint32():
        ref = ((x / 4294967295.0) * k).astype(np.float32)
        y = (x.astype(np.float32) * np.float32(2.0 ** -32)).astype(np.longdouble)
        fma = (x.astype(np.longdouble) * np.longdouble(c) + y).astype(np.float32)
        assert np.array_equal(ref, fma)
        n += x.size
    assert n == 83886081


def _kiss_numpy(state, draws):
    s1, s2, s3, s4, s5 = [np.uint32(x) for x in state]
    out = []
    for _ in range(draws):
        s2 ^= np.uint32(s2 << np.uint32(5))
        s2 ^= np.uint32(s2 >> np.uint32(7))
        s2 ^= np.uint32(s2 << np.uint32(22))
        t = np.int32(np.uint32(s3 + s4 + s5).view(np.int32))
        s3 = s4
        s5 = np.uint32(1 if t < 0 else 0)
        s4 = np.uint32(np.uint32(t.view(np.uint32)) & np.uint32(2147483647))
        s1 = np.uint32(s1 + np.uint32(1411392427))
        x = np.float32(np.uint32(s1 + s2 + s4))
        out.append(np.float32((float(x) / 4294967295.0) * float(np.float32(1) - np.float32(2.0 ** -23))))
    return out


def test_kiss_known_answers():
    """First draws of slot 0 for seed 777, restated in numpy (KissUniform)."""
    st = scenes.seed_states(777)
    with np.errstate(over="ignore"):
        vals = _kiss_numpy(st[:, 0], 8)
    assert all(0.0 <= v < 1.0 for v in vals)
    assert len(set(vals)) == 8
