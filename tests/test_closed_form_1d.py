"""The 1D closed-form restatement (ClosedFormInt, cpab/cpa1d/calcs/ClosedFormInt.py)
against the reference's REF scheme as nStepsODE grows, and its own round trip.
CPU only."""
import numpy as np

from cpabdiffeo_b200.space import Prior, build_space


def _setup(seed=3, nC=20):
    geo = build_space(1, (nC,), "II")
    rng = np.random.default_rng(seed)
    theta = Prior.create(geo, 0.1, 1.0).sample(1, rng)[0]
    A = (geo.B @ theta).reshape(nC, 2)
    return geo, A, rng


def test_closed_form_matches_fine_midpoint(oracle_mod):
    O = oracle_mod
    geo, A, rng = _setup()
    x = rng.uniform(0, 1, 3000)
    T = 1.0
    cf, nf = O.closed_form_1d(A, geo.nC, x, T)
    assert nf == 0
    t = O.tess_struct(1, 2, geo.nCs, geo.incs)
    fine = O.calc_T_simple(t, A, x[:, None], T / 10, 10, 2000)[:, 0]
    assert np.abs(cf - fine).max() < 1e-6


def test_closed_form_round_trip(oracle_mod):
    O = oracle_mod
    geo, A, rng = _setup(5)
    x = rng.uniform(0.01, 0.99, 2000)
    y, _ = O.closed_form_1d(A, geo.nC, x, 1.0)
    z, _ = O.closed_form_1d(-A, geo.nC, y, 1.0)
    assert np.abs(z - x).max() < 1e-9


def test_closed_form_monotone(oracle_mod):
    """A 1D diffeomorphism preserves order."""
    O = oracle_mod
    geo, A, _ = _setup(9)
    x = np.linspace(0, 1, 5001)
    y, _ = O.closed_form_1d(A, geo.nC, x, 1.0)
    assert (np.diff(y) >= -1e-12).all()
    assert y[0] == 0.0 and y[-1] == 1.0
