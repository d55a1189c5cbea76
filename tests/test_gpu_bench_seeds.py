"""The bench's per-rank C3 free data: every seed a multi-GPU run hands to a
rank must give a base shoot that converges, or that rank would stop while the
others wait at the next barrier."""
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parent.parent


def test_rank_seeds_give_converging_base_shoots(engine):
    import pcc

    sys.path.insert(0, str(REPO))
    import bench

    seeds = [bench.rank_seed(bench.C3_SEEDS[0], r) for r in range(8)]
    assert len(set(seeds)) == 8 and seeds[0] == bench.C3_SEEDS[0]
    cfg, _ = bench.workload(seeds[0], 0.1)
    s = engine.solve(pcc.SolveDesc.from_config(cfg))
    st = {}
    for seed in bench.C3_SEEDS:
        _, in0 = bench.workload(seed, 0.1)
        s.shoot(in0, stats=st)  # raises PccError on an IRK failure
        assert st["fail_column"] == -1, seed
