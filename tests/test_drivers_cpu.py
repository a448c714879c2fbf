"""The C++ drivers (hrnn_b200/drivers) take the reference drivers' flags: usage,
defaults, and the errors for missing or unknown options (no GPU needed)."""
import os
import subprocess

import pytest

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "hrnn_b200", "drivers", "bin")


def run(name, *args):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.skip("drivers not built (make -C hrnn_b200/drivers)")
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=60)


@pytest.mark.parametrize("name,flags", [
    ("hrnn_build", ["--base", "--index_path", "--M arg (=16)", "--ef_construction arg (=200)",
                    "--K_knng arg (=500)", "--nn_iters arg (=3)", "--nn_sample arg (=20)", "--num_threads arg (=64)"]),
    ("hrnn_search", ["--index_path", "--query", "--gt", "--k arg (=10)", "--K_prime arg (=500)",
                     "--m arg (=1,3,5,10,20,50)", "--threshold arg (=1)", "--ef_search arg (=200)",
                     "--max_queries arg (=0)", "--max_k_serve arg (=0)"]),
    ("hrnn_dynamic_test", ["--base", "--query", "--gt", "--snapshot", "--oracle_snapshot", "--batch_size arg (=0)",
                           "--K_knng arg (=500)", "--m arg (=50)", "--split arg (=0.5)", "--m_update arg (=0)",
                           "--bidirectional arg (=0)"]),
])
def test_driver_usage(name, flags):
    r = run(name, "--help")
    assert r.returncode == 0
    for f in flags:
        assert f in r.stdout, (name, f)


def test_driver_errors():
    r = run("hrnn_build", "--index_path", "x.idx")
    assert r.returncode == 1 and "'--base' is required" in r.stderr
    r = run("hrnn_search", "--bogus", "1")
    assert r.returncode == 1 and "unrecognised option" in r.stderr
    r = run("hrnn_build", "--base=/nonexistent.fbin", "--index_path", "x.idx")
    assert r.returncode == 1 and "Cannot open: /nonexistent.fbin" in r.stderr
