"""bench.py's launcher (CPU, no GPU work): `--gpus N` outside torchrun runs N
ranks through torch.distributed.run and the line reports n_gpus = N; under
torchrun a WORLD_SIZE that differs from --gpus is refused."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def run(args, env_extra=None):
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, BENCH, *args], capture_output=True, text=True,
                          timeout=240, env=env, cwd=ROOT)


def last_json(out):
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    return json.loads(lines[-1])


def test_gpus_two_spawns_two_ranks():
    r = run(["--gpus", "2", "--dry-run"])
    assert r.returncode == 0, r.stderr
    line = last_json(r.stdout)
    assert line["n_gpus"] == 2 and line["gpus_arg"] == 2


def test_single_rank_dry_run():
    r = run(["--dry-run"])
    assert r.returncode == 0, r.stderr
    assert last_json(r.stdout)["n_gpus"] == 1


def test_world_size_must_match_gpus():
    r = run(["--gpus", "2", "--dry-run"], {"WORLD_SIZE": "3", "RANK": "0"})
    assert r.returncode == 2
    assert "WORLD_SIZE=3" in r.stderr


def test_step_profile_matches_the_timed_kernels_only():
    """The committed step summary gives the issue and L2 figures for the
    kernels it was measured on, and nothing for other kernel choices."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", BENCH)
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    desc = {"cycle_kernel": 0, "cluster_size": 16, "j1_kernel": 1, "replica_group": 4,
            "chains": 2, "j1_site_mode": 1, "j1_fixed_l": 1, "autotune_choice": 4}
    prof = bench.profiled_step(desc)
    assert prof is not None
    assert 1.0 < prof["warp_instructions_per_update"] < 10.0
    assert 10.0 < prof["l2_bytes_per_update"] < 400.0
    assert prof["l2_peak_gbs"] > 1000.0
    cell = bench.profiled_step(dict(desc, j1_site_mode=0))
    assert cell is not None
    assert cell["warp_instructions_per_update"] < prof["warp_instructions_per_update"]
    assert bench.profiled_step(dict(desc, j1_fixed_l=0)) is None
    assert bench.profiled_step(dict(desc, j1_site_mode=3)) is None
