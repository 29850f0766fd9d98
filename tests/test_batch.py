"""The batched executor for scans of uneven size (disorder_b200.batch): a
batch reconstructed by concurrent workers (one context, stream and host
thread each) gives every scan the result of its own single-scan run."""

import numpy as np
import pytest


def test_uneven_specs_and_rectangular_sampling():
    from disorder_b200 import batch, synth
    specs = batch.uneven_specs(32, 4000)
    assert len(specs) == 32 and len({sp["seed"] for sp in specs}) == 32
    assert {s for sp in specs for s in sp["N"]} <= set(batch.SIZES)
    # 96 shots on a grid the 8 x 12 tile does not divide: every shot sampled
    H = synth.random_checkered((128, 160), 96, np.random.default_rng(1), truncate=True)
    counts = np.bincount(H.ravel(), minlength=97)[1:]
    assert counts.min() > 0 and counts.max() - counts.min() <= 16
    # LPT order: costliest first
    order = sorted(specs, key=lambda sp: -batch.cost(sp))
    assert batch.cost(order[0]) >= batch.cost(order[-1])


@pytest.mark.gpu
def test_batch_matches_single_scan_runs():
    from disorder_b200 import batch
    specs = [{"N": (48, 32, 32), "coils": 8, "shots": 16, "seed": 11},
             {"N": (32, 48, 40), "coils": 4, "shots": 32, "seed": 12},
             {"N": (64, 32, 24), "coils": 8, "shots": 16, "seed": 13},
             {"N": (40, 40, 32), "coils": 4, "shots": 16, "seed": 14}]
    runner = batch.BatchRunner(workers=2)
    scans = [batch.build(runner.ctxs[0], sp, n_ell=8) for sp in specs]
    r = runner.run(scans)
    assert not r["failures"], r["failures"]
    assert r["scans_per_s"] > 0 and r["p99_s"] >= r["p50_s"] > 0
    ref = batch.BatchRunner(workers=1)
    for sc, e in zip(scans, r["nrmse"]):
        x, _, _ = batch.reconstruct(ref.ctxs[0], sc)
        xh = x.numpy()
        e1 = float(np.linalg.norm(xh - sc.x_gt_host) / np.linalg.norm(sc.x_gt_host))
        assert abs(e - e1) <= 1e-6 * e1, (sc.spec, e, e1)
        assert np.isfinite(e1) and e1 < 1.0
