"""The standard bench workload at full size (256x128x96, 3.1 M cells) from the
reference reset state, step after step through WAAMTwin, against the CPU
oracle's field hashes (tests/golden/trajectory_standard.json): the same
bits every 500 steps, droplets, quiet tiles, the pipelined and lagged stream
and the population copy included."""
import json
import os
import sys

import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_standard_workload_trajectory_matches_oracle_hashes():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import bench
    from make_trajectory import FIELDS, record
    with open(os.path.join(HERE, "golden", "trajectory_standard.json")) as fh:
        fix = json.load(fh)
    # compare while the oracle's state is finite
    recs = [r for r in fix["records"] if r["nonfinite_T"] == 0]
    assert len(recs) >= 10
    w = dict(bench.WORKLOADS["standard"])
    tw = bench.build_twin(w, torch.device("cuda", 0))
    pos = bench.path_steps(w, tw.grid.dt, recs[-1]["step"])
    want = {r["step"]: r for r in recs}
    for s in range(recs[-1]["step"]):
        tw.step(*pos[s])
        if s + 1 in want:
            got = record(s + 1, tw.grid.state_dict(), tw._n_droplets_fired)
            ref = want[s + 1]
            for k in ("drops", "gas", "read_is_a") + FIELDS:
                assert got[k] == ref[k], (s + 1, k, got[k], ref[k])
    assert tw._n_droplets_fired >= 10
