"""The C++ host driver pyro_run (reference option names) over the C-ABI."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cudacode_b200", "pyro_run")


def test_cli_help_and_bad_option():
    assert os.path.exists(CLI), "build with python -m cudacode_b200.build"
    r = subprocess.run([CLI, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--NumberOfTemperatures" in r.stdout
    r = subprocess.run([CLI, "--no-such-option"], capture_output=True, text=True)
    assert r.returncode == 1 and "unknown option" in r.stderr


@pytest.mark.gpu
def test_cli_matches_python_engine(tmp_path):
    from cudacode_b200.engine import Engine, System, geometric_ladder

    out = tmp_path / "E.dat"
    args = ["--nx", "4", "--NumberOfTemperatures", "6", "--TMin", "0.1", "--TMax", "1.5",
            "--LogScale", "--OverRelaxation", "3", "--McStepsParallelTempering", "1",
            "--ThermalizationSteps", "20", "--NumberOfMeasures", "15", "--Rng", "777",
            "--Heisenberg", "1", "--Output", str(out)]
    r = subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.loadtxt(out)[:, 1:]
    temps = geometric_ladder(0.1, 1.5, 6)
    e = Engine([System(L=4, temperatures=temps)], seed=777, renorm_every=100)
    e.init_random()
    e.tune_cone(0.5, 50, 10, 3)
    for _ in range(20):
        e.cycle(1, 3, True, 1)
    want = []
    for _ in range(15):
        e.cycle(1, 3, True, 1)
        E, _ = e.observables()
        perm = e.permutation()
        want.append(E[perm] / (16 * 64))
    np.testing.assert_allclose(got, np.array(want), rtol=1e-9, atol=1e-12)


@pytest.mark.gpu
def test_cli_anisotropic_model_matches_python_engine(tmp_path):
    from cudacode_b200.engine import (Engine, System, geometric_ladder, reference_exchange,
                                      reference_field, reference_gtensor)

    out = tmp_path / "E.dat"
    J = (-0.09 / 0.29, -0.22 / 0.29, -1.00, 0.0)  # the reference's defaults
    args = ["--nx", "3", "--NumberOfTemperatures", "4", "--TMin", "0.1", "--TMax", "2.0",
            "--LogScale", "--OverRelaxation", "2", "--ThermalizationSteps", "10",
            "--NumberOfMeasures", "8", "--Rng", "99", "--MagneticField", "--Bx", "0",
            "--Bz", "2", "--gxy", "2.4", "--gz", "0.3", "--Magnetization", "--Output", str(out)]
    r = subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got_e = np.loadtxt(out)[:, 1:]
    got_m = np.loadtxt(str(out) + ".magnetization")[:, 1:]
    temps = geometric_ladder(0.1, 2.0, 4)
    e = Engine([System(L=3, temperatures=temps, J1=0.0)], seed=99, renorm_every=100)
    e.set_exchange(reference_exchange(*J), reference_field(2.4, 0.3, [0.0, 0.0, 2.0]))
    e.init_random()
    e.tune_cone(0.5, 50, 10, 2)
    for _ in range(10):
        e.cycle(1, 2, True, 1)
    g = reference_gtensor(2.4, 0.3)
    N = 16 * 27
    want_e, want_m = [], []
    for _ in range(8):
        e.cycle(1, 2, True, 1)
        E, _ = e.observables()
        perm = e.permutation()
        sub = e.sublattice_magnetisation()  # (R, 4, 3)
        Mg = np.einsum("bik,rbk->ri", g, sub)
        want_e.append(E[perm] / N)
        want_m.append((Mg[perm] / N).ravel())
    np.testing.assert_allclose(got_e, np.array(want_e), rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(got_m, np.array(want_m), rtol=1e-9, atol=1e-12)


@pytest.mark.gpu
def test_cli_statistics_files_match_the_oracle(tmp_path):
    """The statistics files of the CLI's measurement loop (measured from
    snapshots while the next cycle runs) against the same chain run by the
    host oracle and measured on the host: the oracle's FP64 energies, order
    parameters and sublattice sums of its spins (the chains are identical bit
    for bit, so the files must agree to FP64 rounding)."""
    from cudacode_b200.engine import (System, geometric_ladder, reference_exchange,
                                      reference_field, reference_gtensor)
    from oracle.binding import Oracle

    args = ["--nx", "3", "--NumberOfTemperatures", "4", "--TMin", "0.2", "--TMax", "2.0",
            "--LogScale", "--OverRelaxation", "1", "--ThermalizationSteps", "5",
            "--NumberOfMeasures", "12", "--Rng", "5", "--MagneticField", "--Bz", "1",
            "--OrderParameters", "--Quadrupole", "--Zaxis", "--ZaxisSum", "--DChiDt",
            "--Magnetization", "--NumberOfRepetitions", "2", "--Output", "series.dat"]
    r = subprocess.run([CLI] + args, capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    for name in ("Energies", "OrderParameters", "dchidt", "Quadrupole", "Sz", "SzSum",
                 "Magnetization"):
        for rep in (0, 1):
            assert (tmp_path / f"{name}{rep}.dat").exists(), (name, rep)
    assert (tmp_path / "series.dat.1").exists()
    temps = geometric_ladder(0.2, 2.0, 4)
    J = (-0.09 / 0.29, -0.22 / 0.29, -1.00, 0.0)
    e = Oracle([System(L=3, temperatures=temps, J1=0.0)], seed=5, renorm_every=100)
    e.set_exchange(reference_exchange(*J), reference_field(1.0, 1.0, [1.0, 0.0, 1.0]))
    e.init_random()
    e.tune_cone(0.5, 50, 10, 1)
    for _ in range(5):
        e.cycle(1, 1, True, 1)
    g = reference_gtensor(1.0, 1.0)
    rows = {k: [] for k in ("E", "op", "q", "sz", "szs", "mag")}
    for _ in range(12):
        e.cycle(1, 1, True, 1)
        E, _ = e.observables()
        perm = e.permutation()  # replica of each temperature
        q = e.order_parameters()[perm]
        spins = e.get_spins()[..., :3].astype(np.float64)      # [replica][site][cell][xyz]
        sub = spins.reshape(len(temps), 4, 4, -1, 3).sum(axis=(1, 3))  # site = 4 f + b
        Mg = np.einsum("bik,rbk->ri", g, sub)[perm]
        rows["E"].append(np.stack([E[perm], E[perm] ** 2], axis=1))
        sq = np.stack([q[:, 0] ** 2, (q[:, 1:3] ** 2).sum(1), (q[:, 3:6] ** 2).sum(1),
                       (q[:, 6:9] ** 2).sum(1), (q[:, 9:12] ** 2).sum(1)], axis=1)
        rows["op"].append(np.concatenate([np.sqrt(sq), sq], axis=1))
        qxx, qxy, qxz, qyy, qyz, qzz = q[:, 12:18].T
        rows["q"].append(np.stack([np.sqrt((2 * qxx - qyy - qzz) ** 2 + 3 * (qzz - qyy) ** 2),
                                   np.sqrt(qxy ** 2 + qxz ** 2 + qyz ** 2),
                                   np.sqrt(qxx ** 2 + qyy ** 2 + qzz ** 2 + qxy ** 2 + qxz ** 2
                                           + qyz ** 2)], axis=1))
        rows["sz"].append(q[:, 19:20])
        rows["szs"].append(q[:, 18:19])
        rows["mag"].append(np.linalg.norm(Mg, axis=1)[:, None])
    for name, key in (("Energies", "E"), ("OrderParameters", "op"), ("Quadrupole", "q"),
                      ("Sz", "sz"), ("SzSum", "szs"), ("Magnetization", "mag")):
        got = np.loadtxt(tmp_path / f"{name}0.dat")
        np.testing.assert_allclose(got[:, 0], temps, rtol=1e-9)
        assert np.all(got[:, 1] == 12)
        want = np.mean(rows[key], axis=0)  # (T, columns)
        np.testing.assert_allclose(got[:, 2::2], want, rtol=1e-9, atol=1e-9, err_msg=name)
