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
            "--Output", str(out)]
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
