"""bench.py's reference arm on the CPU: the contract's JSON line on a small
configuration (no GPU needed: the arm times the CPU oracle port)."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_one_contract_line(tmp_path):
    env = dict(os.environ, SVR_SCENE_CACHE=str(tmp_path / "scenes"))
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "c1",
                          "--steps", "2", "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "ms/view" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"] == {"value": d["value"], "unit": "ms/view", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "view k mod 3" in d["cpu_baseline"]["sample"]
