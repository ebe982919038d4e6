"""The arithmetic contract of one update (include/pyro_math.h), on the host:
Philox4x32-10 known-answer vectors and the accuracy of the engine's own
elementary functions."""
import math

import numpy as np
import pytest

from oracle import binding as orc

# Known-answer vectors published with Random123 (Salmon et al., SC'11) for
# philox4x32 with 10 rounds: (counter, key) -> output.
PHILOX_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(ctr, key, want):
    assert orc.philox(ctr, key).tolist() == want


def ulp_err(got, want):
    want32 = np.float32(want)
    return abs(float(np.float32(got)) - float(want)) / float(np.spacing(np.abs(want32)))


def test_expf_accuracy():
    xs = np.concatenate([-np.logspace(-6, math.log10(86.9), 4000), np.linspace(-1, 0, 1001)])
    worst = max(ulp_err(orc.expf(float(x)), math.exp(float(np.float32(x)))) for x in xs)
    assert worst < 4.0, worst
    assert orc.expf(-90.0) == 0.0
    assert orc.expf(0.0) == 1.0


def test_logf_accuracy():
    xs = np.concatenate([np.logspace(-30, 30, 4000), np.linspace(0.5, 2.0, 1001)])
    worst = 0.0
    for x in xs:
        x32 = float(np.float32(x))
        want = math.log(x32)
        if abs(want) < 1e-3:
            err = abs(orc.logf(x32) - want)
            assert err < 1e-7
            continue
        worst = max(worst, ulp_err(orc.logf(x32), want))
    assert worst < 4.0, worst


def test_sincospif_accuracy():
    for a in np.linspace(0.0, 2.0, 4001, endpoint=False):
        a32 = float(np.float32(a))
        s, c = orc.sincospif(a32)
        assert abs(s - math.sin(math.pi * a32)) < 3e-7
        assert abs(c - math.cos(math.pi * a32)) < 3e-7
        assert abs(s * s + c * c - 1.0) < 1e-6


def test_exp64_accuracy():
    for x in np.concatenate([-np.logspace(-12, math.log10(699), 3000), [0.0]]):
        want = math.exp(x)
        got = orc.exp64(float(x))
        assert abs(got - want) <= 4 * np.spacing(want), (x, got, want)
    assert orc.exp64(-800.0) == 0.0
