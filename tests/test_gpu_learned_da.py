"""What the trained survival classifier gains over the plain scan, under the
method's retirement rule: only probes it marks confidently lost
(p(lost) > 0.98 at the snapshot turn) are retired early; every other probe,
the predicted DA boundary +-2 grid cells and a 2 % random audit are tracked
to the full turn count by the FP64 tracker.  The gain is bounded by the
probes that are alive at the snapshot and lost later: on these error rings
almost every lost probe is lost within a few turns, so the bound -- and the
gain -- is small (well under 1 % of the particle.turns at 20,000 turns).

The network is trained on the GPU (hand-written tcgen05 forward/backward) on
the tracker's own survive/lost labels of training variants and prunes
held-out variants.  The test asserts that the pruned scan tracks fewer
particle.turns than the plain scan of the same probes
(bmad/modules/dynamic_aperture_mod.f90:335-388 is the search it replaces),
reaches the same DA radius within 2 %, retires no probe as surviving, and
that every tracked probe's outcome equals the plain scan's.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_pruned_scan_gain_under_the_retirement_rule():
    from bgt import da, rings
    from bgt import learned_da as LD
    from bgt.mlp import SurvivalMLP
    from bgt.track import Tracker

    lats = rings.error_variants(12, seed=61)
    grid = rings.DAGrid(16, 40, 0.025, (0.0,), 3000)
    early = 8  # the snapshot turn of this small test (64 in the configured scan)
    ys = da.y_scale(rings.TWISS0["beta_a"], rings.TWISS0["beta_b"])
    k2 = (rings.K2_SF, rings.K2_SD)
    pb_tr = LD.setup(Tracker(lats[:8]), lats[:8], grid, k2, yscale=ys)
    pb_te = LD.setup(Tracker(lats[8:]), lats[8:], grid, k2, yscale=ys)
    st = LD.staged_scan(pb_tr, 0, 8, early=early)
    net = SurvivalMLP(max_batch=8192, seed=3)
    raw, lab = LD.training_set(pb_tr, [st], net)
    assert lab.sum() > 20  # probes alive at the snapshot and lost later are in the labels
    LD.train(net, raw, lab, epochs=40, batch=256, lr=2e-3, seed=3)

    plain = da.plain_scan(pb_te.tracker, pb_te.ref, **pb_te.grid())
    pr = LD.pruned_scan(pb_te, net, 0, 4, early=early, p_hi=0.98, p_lo=0.0, boundary_cells=2, seed=5,
                        retune_subset=False)
    surv = plain.survive_turns.reshape(-1)
    plain_surv = surv >= grid.n_turns

    # the rule: nothing retired as surviving; whatever is retired had p > 0.98
    assert pr.n_retired_survive == 0
    retired = ~pr.tracked & ~np.isnan(pr.p_lost)
    assert np.all(pr.p_lost[retired] > 0.98)
    # the gain: fewer particle.turns than the plain scan of the same probes,
    # at most what retiring every probe alive at the snapshot but lost later
    # would save
    late = (surv >= early) & (surv < grid.n_turns)
    bound = plain.particle_turns - int(np.sum(surv[late] - early))
    assert pr.n_retired_lost > 0
    assert bound <= pr.particle_turns < plain.particle_turns
    # same DA radius within 2 %, tracked outcomes equal the plain scan's
    err = da.da_error(pr.radius, plain.radius)
    assert err <= 0.02, err
    assert np.array_equal(pr.survive_label[pr.tracked], plain_surv[pr.tracked])
    print(f"\nLEARNED-DA rule-following: particle.turns pruned {pr.particle_turns} / plain {plain.particle_turns} "
          f"= {pr.particle_turns / plain.particle_turns:.4f} (bound {bound / plain.particle_turns:.4f}), "
          f"retired lost {pr.n_retired_lost}, DA error {err:.4f}, "
          f"wall pruned {pr.wall_s:.2f} s / plain {plain.wall_s:.2f} s")
