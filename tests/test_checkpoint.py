"""Checkpoint / resume (bit-exact continuation), failure detection on
corrupt, truncated, missing or mismatched files, and the reference's
per-temperature configuration files."""
import os

import numpy as np
import pytest

from cudacode_b200.engine import Engine, PyroError, System, geometric_ladder

pytestmark = pytest.mark.gpu

TEMPS = geometric_ladder(0.05, 1.5, 5)


def fresh(L=5, seed=314, **kw):
    e = Engine([System(L=L, temperatures=TEMPS, **kw)], seed=seed, renorm_every=7)
    return e


def test_resume_is_bit_exact(tmp_path):
    path = str(tmp_path / "run.ckp")
    a = fresh()
    a.init_random()
    a.tune_cone(0.5, 4, 3)
    a.cycle(1, 4, True, 6)
    a.save_checkpoint(path)
    a.cycle(1, 4, True, 9)
    b = fresh()
    b.load_checkpoint(path)
    b.cycle(1, 4, True, 9)
    assert np.array_equal(a.get_spins(), b.get_spins())
    assert np.array_equal(a.permutation(), b.permutation())
    assert np.array_equal(a.get_cone(), b.get_cone())
    assert a.sweep_count() == b.sweep_count()


def test_resume_with_learned_move(tmp_path):
    path = str(tmp_path / "tet.ckp")
    a = fresh(L=4)
    a.init_random()
    a.tet_init(seed=9)
    a.cycle_tet(1, 1, 1, True, 3)
    a.save_checkpoint(path)
    a.cycle_tet(1, 1, 1, True, 4)
    b = fresh(L=4)
    b.load_checkpoint(path)
    b.cycle_tet(1, 1, 1, True, 4)
    assert np.array_equal(a.get_spins(), b.get_spins())
    assert np.array_equal(a.tet_weights(), b.tet_weights())


def test_corrupt_truncated_missing_and_mismatched(tmp_path):
    path = str(tmp_path / "c.ckp")
    a = fresh()
    a.init_random()
    a.cycle(1, 1, True, 2)
    a.save_checkpoint(path)
    before = a.get_spins()
    data = open(path, "rb").read()
    bad = bytearray(data)
    bad[len(bad) // 2] ^= 0x40
    open(tmp_path / "flip.ckp", "wb").write(bad)
    open(tmp_path / "short.ckp", "wb").write(data[: len(data) // 3])
    for name in ("flip.ckp", "short.ckp", "missing.ckp"):
        with pytest.raises(PyroError) as ei:
            a.load_checkpoint(str(tmp_path / name))
        assert ei.value.code == -5  # PYRO_ERR_IO
    assert np.array_equal(a.get_spins(), before)  # nothing installed
    other = fresh(L=4)
    with pytest.raises(PyroError) as ei:
        other.load_checkpoint(path)
    assert ei.value.code == -1  # PYRO_ERR_ARG
    other_seed = fresh(seed=1)
    with pytest.raises(PyroError):
        other_seed.load_checkpoint(path)


def test_reference_configuration_files(tmp_path):
    prefix = str(tmp_path / "Conf")
    a = fresh(L=3)
    a.init_random()
    a.cycle(1, 2, True, 5)
    a.save_configurations(prefix)
    a.cycle(1, 2, True, 3)
    a.save_configurations(prefix, append=True)
    spins = a.get_spins()
    perm = a.permutation()  # replica holding each temperature, lowest T first
    n = 16 * 27
    for k in range(5):
        raw = np.fromfile(f"{prefix}{k}.dat", dtype=np.float64)
        assert raw.size == 2 * 3 * n  # two repetitions
        last = raw[3 * n:].reshape(n, 3)
        rep = perm[4 - k]  # k = 0 is the highest temperature
        np.testing.assert_array_equal(last.astype(np.float32), spins[rep, :, :, :3].reshape(n, 3))
    b = fresh(L=3)
    b.read_configurations(prefix, repetition=1)
    # b has the identity permutation: replica t holds temperature t
    np.testing.assert_array_equal(b.get_spins(), spins[perm])
    with pytest.raises(PyroError):
        b.read_configurations(prefix, repetition=2)
