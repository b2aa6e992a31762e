"""The discrete adjoint on the GPU: its gradient against the tangent-linear
reference (the oracle on dual numbers, same frozen dt sequence) and against
central differences of the GPU forward, for random directions in the bed and
the Manning field; and the same gradient whatever the checkpoint interval."""
import numpy as np
import pytest

from tlm import tlm_misfit

pytestmark = pytest.mark.gpu


def case(swe, nx=40, ny=30, steps=30, seed=21):
    from water_simulator_b200 import workloads
    c = workloads.adjoint_case(nx=nx, ny=ny, dx=10.0, n_gauges=6, seed=seed, hump=0.4)
    # observations from the perturbed bed
    truth = swe.MisfitAdjoint(nx, ny, 10.0, c["b_true"], c["eta0"], manning_field=c["n"], gauges=c["gauges"],
                              steps=steps, checkpoint_every=7)
    _, eta = truth.forward()
    truth.close()
    return c, eta


def gradient(swe, c, obs, steps, every=7):
    adj = swe.MisfitAdjoint(c["nx"], c["ny"], c["dx"], c["b"], c["eta0"], manning_field=c["n"], gauges=c["gauges"],
                            steps=steps, checkpoint_every=every)
    adj.set_observations(obs)
    J, _ = adj.forward()
    gb, gn = adj.backward()
    dts = adj.dt_sequence()
    return adj, J, gb, gn, dts


def test_adjoint_matches_tangent_linear(swe):
    steps = 30
    c, obs = case(swe, steps=steps)
    adj, J, gb, gn, dts = gradient(swe, c, obs, steps)
    rng = np.random.default_rng(1)
    for trial in range(4):
        db = rng.normal(0, 1, c["b"].shape)
        dn = rng.normal(0, 1e-3, c["n"].shape) if trial >= 2 else np.zeros(c["n"].shape)
        Jt, dJ, dts_t = tlm_misfit(c, c["b"], c["n"], db, dn, steps, obs)
        assert abs(Jt - J) <= 1e-12 * abs(J)
        got = float(np.dot(gb, db.reshape(-1)) + np.dot(gn, dn.reshape(-1)))
        assert abs(got - dJ) <= 1e-8 * abs(dJ), (trial, got, dJ)
    assert np.all(gb.reshape(c["ny"] + 4, c["nx"] + 4)[:2] == 0)          # ghosts carry no gradient
    adj.close()


def test_adjoint_against_central_differences(swe):
    steps = 30
    c, obs = case(swe, steps=steps, seed=22)
    adj, J, gb, gn, dts = gradient(swe, c, obs, steps)
    rng = np.random.default_rng(2)

    def J_at(b, n):
        f = swe.MisfitAdjoint(c["nx"], c["ny"], c["dx"], b, c["eta0"], manning_field=n, gauges=c["gauges"],
                              steps=steps, checkpoint_every=steps)
        f.set_observations(obs)
        f.dt_sequence(fixed=dts)
        v, _ = f.forward()
        f.close()
        return v

    for trial in range(20):
        db = rng.normal(0, 1, c["b"].shape)
        dn = rng.normal(0, 1e-3, c["n"].shape)
        want = float(np.dot(gb, db.reshape(-1)) + np.dot(gn, dn.reshape(-1)))
        errs = []
        for eps in (1e-4, 1e-5, 1e-6, 1e-7):
            fd = (J_at(c["b"] + eps * db, c["n"] + eps * dn) - J_at(c["b"] - eps * db, c["n"] - eps * dn)) / (2 * eps)
            errs.append(abs(fd - want) / abs(want))
        assert min(errs) <= 1e-5, (trial, errs)
    adj.close()


def test_gradient_independent_of_checkpointing(swe):
    steps = 23
    c, obs = case(swe, steps=steps, seed=23)
    ref = None
    for every in (1, 5, 23):
        adj, J, gb, gn, _ = gradient(swe, c, obs, steps, every)
        if ref is None:
            ref = (gb, gn)
        else:
            assert np.array_equal(gb, ref[0]) and np.array_equal(gn, ref[1])
        adj.close()


def test_gauges_sharing_a_cell(swe):
    """Gauges may repeat a cell: their contributions add in gauge order."""
    steps = 20
    c, _ = case(swe, steps=steps, seed=24)
    g = np.asarray(c["gauges"], dtype=np.int32)
    c["gauges"] = np.concatenate([g, g[:2], g[:1]]).astype(np.int32)
    rng = np.random.default_rng(3)
    obs = rng.normal(2.0, 0.05, (steps, len(c["gauges"])))
    adj, J, gb, gn, dts = gradient(swe, c, obs, steps)
    db = rng.normal(0, 1, c["b"].shape)
    dn = rng.normal(0, 1e-3, c["n"].shape)
    Jt, dJ, _ = tlm_misfit(c, c["b"], c["n"], db, dn, steps, obs)
    assert abs(Jt - J) <= 1e-12 * abs(J)
    got = float(np.dot(gb, db.reshape(-1)) + np.dot(gn, dn.reshape(-1)))
    assert abs(got - dJ) <= 1e-8 * abs(dJ), (got, dJ)
    adj.close()


BOUNDARY_CASES = {
    "outflow_we": {"west": "outflow", "east": "outflow"},
    "periodic_all": {"west": "periodic", "east": "periodic", "south": "periodic", "north": "periodic"},
    "flather_west": {"west": ("flather", 2.05, 0.0), "east": "outflow"},
    "flather_sn_periodic_we": {"south": ("flather", 2.0, 0.01), "north": ("flather", 1.95, -0.02),
                               "west": "periodic", "east": "periodic"},
    "mixed": {"east": ("flather", 2.0, 0.0), "south": "outflow", "north": "periodic"},
    "tide_west": {"west": ("tide", 2.0, [0.3, 0.1], [2 * 3.141592653589793 / 600, 2 * 3.141592653589793 / 250],
                           [0.0, 40.0], 0.05), "east": "outflow"},
}


@pytest.mark.parametrize("name", list(BOUNDARY_CASES))
def test_adjoint_boundaries_match_tangent_linear(swe, name):
    """Outflow, periodic and Flather sides, constant or tidal
    (src/swe.mjs:1026-1126): the forward equals the oracle's, the gradient
    its tangent-linear model."""
    from water_simulator_b200 import workloads
    bcs = BOUNDARY_CASES[name]
    steps, nx, ny = 24, 40, 30
    c = workloads.adjoint_case(nx=nx, ny=ny, dx=10.0, n_gauges=6, seed=31, hump=0.4)
    kw = dict(manning_field=c["n"], gauges=c["gauges"], steps=steps, checkpoint_every=7, boundaries=bcs)
    truth = swe.MisfitAdjoint(nx, ny, 10.0, c["b_true"], c["eta0"], **kw)
    _, obs = truth.forward()
    truth.close()
    adj = swe.MisfitAdjoint(nx, ny, 10.0, c["b"], c["eta0"], **kw)
    adj.set_observations(obs)
    J, _ = adj.forward()
    gb, gn = adj.backward()
    rng = np.random.default_rng(5)
    for trial in range(3):
        db = rng.normal(0, 1, c["b"].shape)
        dn = rng.normal(0, 1e-3, c["n"].shape) if trial else np.zeros(c["n"].shape)
        Jt, dJ, _ = tlm_misfit(c, c["b"], c["n"], db, dn, steps, obs, bcs=bcs)
        assert abs(Jt - J) <= 1e-12 * abs(J), (name, Jt, J)
        got = float(np.dot(gb, db.reshape(-1)) + np.dot(gn, dn.reshape(-1)))
        assert abs(got - dJ) <= 1e-8 * abs(dJ), (name, trial, got, dJ)
    g2 = gb.reshape(ny + 4, nx + 4)
    assert np.all(g2[:2] == 0) and np.all(g2[-2:] == 0) and np.all(g2[:, :2] == 0) and np.all(g2[:, -2:] == 0)
    adj.close()


def test_adjoint_boundary_refusals(swe):
    c = swe.MisfitAdjoint(8, 8, 10.0, np.zeros(144), 1.0, gauges=[50], steps=2)
    with pytest.raises(ValueError):
        c.set_boundary("west", "sponge")
    with pytest.raises(KeyError):
        c.set_boundary("up", "reflect")
    c.close()
