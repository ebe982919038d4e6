"""The engine's counter-based Philox4x32-10 (include/pyro_math.h) against
cuRAND's Philox generator output for output: curand_init(seed, subsequence,
0) followed by curand4 draws block i = Philox(counter (i, 0, subsequence),
key seed). The update contract then consumes these words as documented
(uniforms from the top 24 bits)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import binding as orc

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.gpu
def test_philox_matches_curand(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "curand_philox")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2",
                    os.path.join(HERE, "curand_philox.cu"), "-o", exe], check=True)
    for seed, sub in [(0, 0), (12345, 0), (0xDEADBEEFCAFEF00D, 7), (56081376, 2 ** 33 + 5)]:
        out = subprocess.run([exe, str(seed), str(sub), "64"], capture_output=True, text=True,
                             check=True).stdout.split("\n")
        got = np.array([[int(x) for x in line.split()] for line in out if line.strip()],
                       dtype=np.uint64)
        key = [seed & 0xFFFFFFFF, seed >> 32]
        for i in range(64):
            ctr = [i, 0, sub & 0xFFFFFFFF, sub >> 32]
            np.testing.assert_array_equal(orc.philox(ctr, key).astype(np.uint64), got[i],
                                          err_msg=f"seed {seed} subsequence {sub} draw {i}")
