"""The benchmark's sharded path (`bench.py --sharded`: the multi-patch
workloads through drnum_b200.shard with compact shadows and the exchange in
the step's hook, on one GPU as a group of one) runs end to end and prints
its line."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_sharded_path_runs_on_one_gpu(tmp_path):
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--n", "64", "--steps", "2", "--warmup", "3",
           "--no-cpu-baseline", "--sharded", "--workload-scale", "0.25", "--clock-dir", str(tmp_path)]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["gpu_launches"] > 0 and line["value"] > 0
    sh = line["sharded"]
    assert set(sh) == {"jet", "sphere", "tiled"}
    for name, w in sh.items():
        assert w["value"] > 0 and w["ranks"] == 1 and w["scaling"] == "strong", name
        assert w["exchange_bytes_per_step_max_rank"] == 0.0, name      # a group of one sends nothing
        assert 1.0 <= w["device_cells_fraction_of_grid"] < 1.6, name    # rows padded to 16 bytes
