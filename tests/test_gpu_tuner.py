"""The launch tuner changes no result: while it cycles through block shapes and carveouts, every
call equals the same call with the tuner off, bit for bit, on the first-init and the weak-texture
(APD, edges, labels) paths; afterwards each tuned kernel has kept one setting."""
import numpy as np
import pytest

import dpe_b200 as D
import helpers as h

pytestmark = pytest.mark.gpu


def _same(a, b):
    for k in ("plane", "weak", "views", "costs"):
        assert np.array_equal(a[k], b[k], equal_nan=True), k


def test_tuner_changes_no_result():
    sc = h.S.make_scene("small_weak", seed=2)
    ref = 1
    images, cams, _ = h.view_inputs(sc, ref)
    p0 = h.first_init_params(sc, len(images))
    c = D.Context(0)
    try:
        c.set_autotune(False)
        base0 = c.pm_run(images, cams, p0, seed=41)
        state, weak = h.post_process(base0["plane"], base0["weak"], p0.depth_min, p0.depth_max)
        edge, low, label = h.synthetic_edges(sc.gray[ref])
        p1 = h.refine_params(sc, len(images), level=1, state=D.REFINE_INIT, geom=False)
        kw = dict(plane_in=state, views_in=np.ascontiguousarray(base0["views"]), weak_in=weak, edge=edge, edge_low=low,
                  label=label, seed=51)
        assert (weak == D.WEAK).mean() > 0.02
        base1 = c.pm_run(images, cams, p1, **kw)
        c.set_autotune(True)
        for _ in range(14):  # more than 2 rounds of the 5 block shapes and the 4 carveouts (both calls tune)
            _same(c.pm_run(images, cams, p0, seed=41), base0)
            _same(c.pm_run(images, cams, p1, **kw), base1)
        table = c.tuning()
    finally:
        c.close()
    kept = {e["kernel"]: e for e in table if e["chosen"] >= 0}
    print({k: (e["block"], e["carveout"], e["mean_ms"]) for k, e in kept.items()})
    for k in ("k_random_init", "k_strong_update"):
        assert k in kept, k
    assert all(e["block"][0] * e["block"][1] <= 128 for e in kept.values())
