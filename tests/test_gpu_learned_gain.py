"""What the trained network gains over the method without it.

The same budget truncation is run twice on held-out angle draws of the 8x8
lattice circuit (N = 64, 20 layers, depolarizing 1e-3, weight cap 12, plain
threshold 1e-5 per merge): once ranking the live terms by the network trained on
the engine's own labels, once ranking them by |c| (the reference's
AdaptiveTruncation).  At budgets of 5-40 % of the plain run's peak, the network's
error against the plain run (no budget) must be less than half the |c| ranking's,
summed over the budgets.  (Measured on the full protocol: a median 30x lower
error at equal budget.)"""
import pytest

import pauliprop as pp
from pauliprop import learned as L

pytestmark = pytest.mark.gpu


def test_network_beats_coefficient_ranking():
    lat = L.Lattice(8, 8, 20)
    t_base = 1e-5
    train = L.angle_draws(2, seed=41)
    X, T, _ = L.training_set(lat, train, (6, 10, 14), 1500, t_base, 1e-12)
    mlp = pp.MLP(L.init_params(0))
    mlp.load_data(X, T)
    losses = mlp.train(1500, batch=2048, lr=1e-3, seed=0)
    assert losses[-20:].mean() < 0.1 * losses[:5].mean()
    draw = L.angle_draws(1, seed=42)[0]
    e_ref, _, peak = L.run_plain(lat, draw, t_base)
    err_net, err_c = 0.0, 0.0
    for frac in (0.05, 0.1, 0.2, 0.4):
        B = int(frac * peak)
        err_net += abs(L.run_learned(lat, draw, mlp, B, t_base)[0] - e_ref)
        err_c += abs(L.run_learned(lat, draw, None, B, t_base)[0] - e_ref)
    assert err_net < 0.5 * err_c, (err_net, err_c)
