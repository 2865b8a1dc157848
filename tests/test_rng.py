"""The chains' RNG and exponential (brain-match_b200/csrc/bm_rng.hpp), as
compiled for the CPU: Philox4x32-10 known-answer vectors of the published
algorithm, and the error of the project's exp against the C library's."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle_bind import oracle_lib


def philox(ctr, key):
    L = oracle_lib()
    L.orc_philox.restype = None
    L.orc_philox.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    c = np.array(ctr, np.uint32)
    k = np.array(key, np.uint32)
    o = np.zeros(4, np.uint32)
    L.orc_philox(c.ctypes.data, k.ctypes.data, o.ctypes.data)
    return [int(x) for x in o]


@pytest.mark.parametrize("ctr,key,expected", [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
])
def test_philox4x32_10_known_answers(ctr, key, expected):
    assert philox(ctr, key) == expected


def test_exp_error_bound():
    L = oracle_lib()
    L.orc_exp.restype = C.c_double
    L.orc_exp.argtypes = [C.c_double]
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-700, 0, 20000), rng.uniform(-1, 1, 20000), rng.uniform(0, 700, 5000),
                         [0.0, -0.0, 1e-300, -1e-300, math.log(2), -math.log(2), -708.0, 708.0]])
    worst = 0.0
    for x in xs:
        got = L.orc_exp(float(x))
        ref = math.exp(float(x))
        ulp = math.ulp(ref) if ref > 0 else 5e-324
        worst = max(worst, abs(got - ref) / ulp)
    assert worst <= 2.0, worst
    assert L.orc_exp(0.0) == 1.0
    assert L.orc_exp(-800.0) == 0.0
    assert math.isinf(L.orc_exp(800.0))
