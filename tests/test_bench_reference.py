"""bench.py's reference arm on the CPU: it runs the oracle (the reference path's C++ restatement)
with the oracle's own builder, never loads libbvhcuda, prints one line with the engine arm's
metric, unit and config, and traces the whole workload it names."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "1", "--tubular", "200", "--radial", "50",
        "--rays-log2", "14", "--camera", "128"]

CODE = """
import runpy, sys
sys.argv = ["bench.py"] + {args!r}
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("LOADED", "libbvhcuda" in maps, "liboracle" in maps)
"""


def test_reference_arm_runs_the_oracle_alone():
    res = subprocess.run([sys.executable, "-c", CODE.format(args=ARGS)], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    line = json.loads(lines[0])
    assert res.stdout.strip().splitlines()[-1] == "LOADED False True"
    sys.path.insert(0, str(ROOT))
    import bench

    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT and line["higher_is_better"] is True
    n_rays = (1 << 14) + 128 * 128
    assert line["config"] == bench.headline_config(200 * 50 * 2, n_rays, 1)
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"] > 0
    assert "both whole ray sets" in line["cpu_baseline"]["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
