"""Host-side helpers of bench.py (no GPU).

The serving sample checks every request against the exact levels of the
transverse-field Ising chain from its free-fermion form; that closed form is
pinned here against exact diagonalisation of the same MPO.
"""
import importlib.util
import os

import pytest

from oracle import ed, mpo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("n", [2, 3, 6, 9, 10])
@pytest.mark.parametrize("lam", [0.5, 1.0, 1.37])
def test_tfim_exact_levels_match_ed(bench, n, lam):
    w, _ = ed.lowest_levels(mpo.transverse_ising_ferro(n, lam), 4)
    ex = bench.tfim_exact_levels(n, lam, 4)
    assert len(ex) == 4
    assert max(abs(a - b) for a, b in zip(w, ex)) < 1e-12 * n


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` times the CPU restatement on the host and prints
    one JSON line with the same metric and unit as the GPU arm."""
    import json
    import subprocess
    import sys

    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "sweeps/s" and line["value"] > 0
    assert line["metric"].startswith("sweeps/s @N=100")
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["higher_is_better"] is True
