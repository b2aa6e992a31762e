"""The tangent-linear reference itself (CPU): its directional derivative of
the gauge misfit against central differences on the oracle with the same
frozen dt sequence, and its value part against the plain oracle."""
import numpy as np

from tlm import tlm_misfit, oracle_misfit


def small_case():
    import __graft_entry__
    __graft_entry__.load_package()
    from water_simulator_b200 import workloads
    return workloads.adjoint_case(nx=24, ny=18, dx=10.0, n_gauges=5, seed=11, hump=0.4)


def test_tlm_matches_central_differences():
    case = small_case()
    steps = 25
    rng = np.random.default_rng(0)
    obs = rng.normal(2.0, 0.05, (steps, len(case["gauges"])))
    for trial in range(3):
        db = rng.normal(0, 1, case["b"].shape)
        dn = rng.normal(0, 1e-3, case["n"].shape) if trial == 2 else np.zeros(case["n"].shape)
        J, dJ, dts = tlm_misfit(case, case["b"], case["n"], db, dn, steps, obs)
        assert J == oracle_misfit(case, case["b"], case["n"], steps, obs, dts)
        # A perturbation that crosses a limiter or wet/dry switch is not a
        # derivative; the check takes the step size that stays clear of one.
        errs = []
        for eps in (1e-4, 1e-5, 1e-6, 1e-7):
            Jp = oracle_misfit(case, case["b"] + eps * db, case["n"] + eps * dn, steps, obs, dts)
            Jm = oracle_misfit(case, case["b"] - eps * db, case["n"] - eps * dn, steps, obs, dts)
            errs.append(abs((Jp - Jm) / (2 * eps) - dJ) / abs(dJ))
        assert min(errs) <= 1e-5, (trial, errs)


def test_tlm_with_open_boundaries_matches_central_differences():
    """The same with outflow, periodic and Flather sides (constant and tidal)."""
    case = small_case()
    steps = 20
    rng = np.random.default_rng(4)
    obs = rng.normal(2.0, 0.05, (steps, len(case["gauges"])))
    tide = ("tide", 2.0, [0.3, 0.1], [2 * np.pi / 600, 2 * np.pi / 250], [0.0, 40.0], 0.05)
    for bcs in ({"west": ("flather", 2.05, 0.0), "east": "outflow", "south": "periodic", "north": "periodic"},
                {"south": ("flather", 1.95, -0.02), "north": "outflow", "west": "periodic", "east": "periodic"},
                {"west": tide, "east": "outflow"}):
        db = rng.normal(0, 1, case["b"].shape)
        dn = rng.normal(0, 1e-3, case["n"].shape)
        J, dJ, dts = tlm_misfit(case, case["b"], case["n"], db, dn, steps, obs, bcs=bcs)
        assert J == oracle_misfit(case, case["b"], case["n"], steps, obs, dts, bcs=bcs)
        errs = []
        for eps in (1e-4, 1e-5, 1e-6, 1e-7):
            Jp = oracle_misfit(case, case["b"] + eps * db, case["n"] + eps * dn, steps, obs, dts, bcs=bcs)
            Jm = oracle_misfit(case, case["b"] - eps * db, case["n"] - eps * dn, steps, obs, dts, bcs=bcs)
            errs.append(abs((Jp - Jm) / (2 * eps) - dJ) / abs(dJ))
        assert min(errs) <= 1e-5, (bcs, errs)
