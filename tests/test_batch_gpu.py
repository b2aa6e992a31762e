"""The batched ensemble: every basin bit-identical to running it alone, for
any tile schedule, and the autotuner leaves the state as it found it."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(64, 70), (130, 64), (200, 90), (90, 300), (33, 17), (121, 5), (250, 40), (7, 130),
         (64, 64), (300, 120), (1, 40), (45, 1)]


def basins(swe, tide_period=300.0):
    from water_simulator_b200 import workloads
    out = []
    for q, (nx, ny) in enumerate(SIZES):
        b = workloads.bump_bed(nx, ny, 5.0, seed=50 + q)
        out.append({"nx": nx, "ny": ny, "dx": 5.0, "b": b, "eta0": 2.0,
                    "manning": 0.0 if q % 3 == 0 else 0.015 + 0.002 * q,
                    "tide": {"msl": 2.0, "amp": [0.3], "omega": [2 * math.pi / (tide_period * (1 + q / 7))],
                             "phase_deg": [10.0 * q]}})
    return out


def single(swe, bs):
    sim = swe.ShallowWater(nx=bs["nx"], ny=bs["ny"], dx=bs["dx"], bed=bs["b"], eta0=bs["eta0"],
                           manning=bs["manning"])
    t = bs["tide"]
    periods = {"X": 2 * math.pi / t["omega"][0] / 3600}
    tide = swe.Tide({"X": [t["amp"][0], t["phase_deg"][0]]}, msl=t["msl"], periods_hours=periods)
    tide.terms[0]["omega"] = t["omega"][0]          # the exact double the ensemble was given
    sim.boundaries = {"west": swe.flather(tide.signal())}
    return sim


def test_each_basin_matches_single_grid(swe):
    bs = basins(swe)
    ens = swe.Ensemble(bs)
    ens.run(40)
    for q, b in enumerate(bs):
        sim = single(swe, b)
        assert sim.run(40) == 40
        for f in ("h", "hu", "hv"):
            assert np.array_equal(ens.field(q, f), sim.field(f)), (q, f)
        assert ens.t(q) == sim.t and ens.steps(q) == 40
        sim.close()
    ens.close()


@pytest.mark.parametrize("sched", [dict(rows=16, ctas=0, order=1), dict(rows=64, ctas=148, order=2),
                                   dict(rows=24, ctas=37, order=0), dict(rows=0, ctas=0, order=2),
                                   dict(rows=0, ctas=97, order=1), dict(rows=32, ctas=0, order=0)])
def test_schedule_does_not_change_results(swe, sched):
    bs = basins(swe)
    ref = swe.Ensemble(bs)
    ref.run(21)
    ens = swe.Ensemble(bs)
    ens.set_schedule(**sched)
    ens.run(21)
    for q in range(len(bs)):
        for f in ("h", "hu", "hv"):
            assert np.array_equal(ens.field(q, f), ref.field(q, f)), (sched, q, f)
    ref.close()
    ens.close()


def test_autotune_keeps_state(swe):
    bs = basins(swe)
    ens = swe.Ensemble(bs)
    ens.run(5)
    before = [[ens.field(q, f) for f in ("h", "hu", "hv")] for q in range(len(bs))]
    t_before = [ens.t(q) for q in range(len(bs))]
    res = ens.autotune(trial_steps=2)
    assert res["rows"] in (0, 16, 24, 32, 48, 64) and res["order"] in (0, 1, 2)
    for q in range(len(bs)):
        assert ens.t(q) == t_before[q]
        for k, f in enumerate(("h", "hu", "hv")):
            assert np.array_equal(ens.field(q, f), before[q][k])
    # and it still steps like a fresh ensemble after the tuning
    ens.run(7)
    ref = swe.Ensemble(bs)
    ref.run(12)
    for q in range(len(bs)):
        assert np.array_equal(ens.field(q, "h"), ref.field(q, "h"))
    ens.close()
    ref.close()


@pytest.mark.parametrize("sched", [dict(rows=0, ctas=0, order=0), dict(rows=0, ctas=148, order=1),
                                   dict(rows=0, ctas=7, order=2)])
def test_queue_launch_matches_phase_launches(swe, sched):
    """One persistent launch per step over the work queue gives every basin
    the same bits as a launch per phase, for any grid and tile order (a
    7-CTA grid makes nearly every item wait on the one before it)."""
    bs = basins(swe)
    ref = swe.Ensemble(bs)
    ref.run(23)
    ens = swe.Ensemble(bs)
    ens.set_schedule(**sched)
    ens.set_launch("queue")
    assert ens.launch == "queue"
    ens.run(23)
    ens.synchronize()
    for q in range(len(bs)):
        for f in ("h", "hu", "hv"):
            assert np.array_equal(ens.field(q, f), ref.field(q, f)), (sched, q, f)
        assert ens.t(q) == ref.t(q) and ens.steps(q) == 23
    ref.close()
    ens.close()


def test_queue_wait_that_nothing_ends_times_out(swe):
    """A basin whose prepare is never marked done (the test hook): its next
    phase waits until the limit (50 ms), the step is dropped, and the host
    reads SWE_ETIMEOUT; the GPU stays usable and the hook off runs again."""
    import time
    bs = basins(swe)
    ens = swe.Ensemble(bs)
    ens.set_launch("queue")
    ens.set_wait_limit(0.05)
    ens.debug_hold(3)
    t0 = time.perf_counter()
    ens.run(2)
    with pytest.raises(swe.SweError) as e:
        ens.synchronize()
    assert e.value.code == -4                          # SWE_ETIMEOUT
    assert time.perf_counter() - t0 < 30
    ens.synchronize()                                  # reported once, then cleared
    ens.close()
    fresh = swe.Ensemble(bs)
    fresh.set_launch("queue")
    fresh.run(3)
    fresh.synchronize()
    assert all(fresh.steps(q) == 3 for q in range(len(bs)))
    fresh.close()
