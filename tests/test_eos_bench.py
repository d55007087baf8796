"""The reference's EOS bench (libs/cuda/src/eos_bench.cu): inputs T, S, z as
functions of the 1-based cell index, the checksum = sum of every max(1, n/1000)-th
result. The reference records the checksums its NumPy, gfortran, nvfortran and
CUDA builds agree on (docs/25_kernel_matrix.md:372-373 at n = 3e7, :395-397 at
n = 3e6). The oracle reproduces them (CPU); eos_bench_b200 prints the oracle's
checksum (GPU)."""

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import ocean_oracle as orc

ROOT = Path(__file__).resolve().parents[1]
RECORDED = {3_000_000: {"linear": "-8.905003e+02", "seos": "-1.057236e+03", "teos10": "1.036620e+06"},
            30_000_000: {"linear": "-8.861232e+02", "seos": "-1.053170e+03", "teos10": "1.036636e+06"}}


def sampled_inputs(n):
    i0 = np.arange(0, n, max(1, n // 1000), dtype=np.int64)  # 0-based cells in the checksum
    T = 5.0 + 15.0 * np.mod(i0 + 1, 977).astype(np.float64) / 977.0
    S = 33.0 + 3.0 * np.mod(i0 + 1, 733).astype(np.float64) / 733.0
    z = 5000.0 * np.mod(i0 + 1, 521).astype(np.float64) / 521.0
    return T, S, z


def oracle_checksum(n, kind):
    T, S, z = sampled_inputs(n)
    if kind == "teos10":
        rho = orc.rho_teos10(T, S, z)
    else:
        rho = orc.rho_anomaly(kind, T, S, z, 1025.0, 2.0e-4, 7.4e-4, 10.0, 35.0)
    chk = 0.0
    for v in rho:  # index order, one by one, as the bench sums
        chk += float(v)
    return chk


@pytest.mark.parametrize("n", sorted(RECORDED))
@pytest.mark.parametrize("kind", ("linear", "seos", "teos10"))
def test_oracle_reproduces_recorded_checksums(n, kind):
    assert f"{oracle_checksum(n, kind):.6e}" == RECORDED[n][kind]


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ("linear", "seos", "teos10"))
def test_eos_bench_executable(kind):
    n = 3_000_000
    exe = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "bin" / "eos_bench_b200"
    proc = subprocess.run([str(exe), str(n), kind, "5"], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr
    first = proc.stdout.splitlines()[0]
    fields = dict(re.findall(r"(\w+)=\s*(\S+)", first))
    assert fields["eos"] == kind and int(fields["n"]) == n
    assert float(fields["checksum"]) == float(f"{oracle_checksum(n, kind):.6e}")
    assert f"{float(fields['checksum']):.6e}" == RECORDED[n][kind]
    assert float(fields["wall"]) > 0.0
