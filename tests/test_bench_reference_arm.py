"""bench.py's reference arm (--impl reference) runs on the host alone: the
reference's own CPU simulator (oracle/_ref) times the same workload and
prints one JSON line with the contract's keys. Checked here at 16 qubits,
one step."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libkate_ref.so")


def _run(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--nqubits", "16",
                        "--steps", "1", "--warmup", "0", *args], capture_output=True, text=True, timeout=300,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref/libkate_ref.so not built")
@pytest.mark.parametrize("workload,metric,higher", [("layers", "16q layers/s", True),
                                                     ("qulacs", "QulacsBench 16q wall time", False)])
def test_reference_arm_prints_the_contract_line(workload, metric, higher):
    d = _run("--workload", workload)
    assert d["impl"] == "reference" and d["metric"] == metric
    assert d["value"] > 0 and d["higher_is_better"] is higher
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["steps"] == 1 and d["warmup"] == 0 and d["config"]["nqubits"] == 16


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref/libkate_ref.so not built")
def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--nqubits", "12",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=ROOT,
                       env=env)
    assert r.returncode == 0 and r.stdout.strip() == ""
