"""
bench.py's command-line contract on the host: the reference arm of the
surrogate-network configuration (no counterpart in sasmodels) prints one
`unavailable` line and exits 0; the MLP flop count matches the network's
shape; the measured-peak reader falls back when the file is absent.
"""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_mlp_reference_arm_is_unavailable():
    proc = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--config", "mlp",
                           "--impl", "reference"], capture_output=True, text=True, cwd=ROOT,
                          timeout=300)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [l for l in proc.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and "unavailable" in line


def test_mlp_flops_and_peak_reader(tmp_path, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    # 16 -> 256, three 256 -> 256, 256 -> 1, two flops per multiply-add
    assert bench.MLP_FLOPS_PER_ROW == 2*(16*256 + 3*256*256 + 256) == 401920
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.bf16_peak() == (1590.0, "of fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"bf16_tflops": 1641.8}))
    peak, source = bench.bf16_peak()
    assert peak == 1641.8 and source.startswith("of measured")
