"""The deterministic log is monotone over every positive float: the crossing search's exact node test
(PixelProc::may_fire_exact) bounds ln(I) over a node by its values at the node's ends, which needs it."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_log_f_is_monotone(tmp_path):
    exe = tmp_path / "log_monotone"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-pthread",
                    f"-I{ROOT / 'ballasim_b200' / 'csrc'}", str(ROOT / "tests" / "native" / "log_monotone.cc"),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=600)
    assert int(out.stdout.strip()) == 0
