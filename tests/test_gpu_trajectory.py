"""Bench workloads at full size from the reference reset state, step after step
through WAAMTwin, against the CPU oracle's field hashes
(tests/golden/trajectory_<workload>.json): the same bits at every checkpoint
-- the standard workload (256x128x96, 3.1 M cells) every 500 steps through
step 9,000, droplets, quiet tiles, the pipelined and lagged stream and the
population copy included; the small one (64x32x32) every 250 steps through
step 2,000."""
import json
import os
import sys

import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.parametrize("workload,min_records,min_drops", [("standard", 18, 17),
                                                             ("small", 8, 0)])
def test_workload_trajectory_matches_oracle_hashes(workload, min_records, min_drops):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import bench
    from make_trajectory import FIELDS, fixture_path, record
    with open(fixture_path(workload)) as fh:
        fix = json.load(fh)
    # compare while the oracle's state is finite
    recs = [r for r in fix["records"] if r["nonfinite_T"] == 0]
    assert len(recs) >= min_records
    w = dict(bench.WORKLOADS[workload])
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
    assert tw._n_droplets_fired >= min_drops
