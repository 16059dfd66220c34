"""CPU: bench.py's reference arm prints one JSON line of the bench contract.

`bench.py --impl reference` times the CPU restatement of the reference's fixed-point datapath (the C
restatement of mpfs/host/silicon_emulator.py:226-249, one whole Centerfield-shaped frame per step on the
host threads) and checks the first frame's CRC against the unmodified reference emulator's CRC of the
same frame.  No GPU is involved; the line must carry the same metric, unit and direction as the GPU arm,
a cpu_baseline describing the run and an e2e block with no host-device bytes.
"""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"].startswith("ms per 8192^2 PFA frame") and d["unit"] == "ms/frame"
    assert d["higher_is_better"] is False and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] >= 3
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert d["config"]["workload"] == "centerfield_5634x4319"
    assert d["crc_equals_reference_emulator"] is True
