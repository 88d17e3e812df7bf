"""The learned K=4 depth operator (no counterpart in the reference).

* gradients of the GPU training kernels against the FP64 CPU restatement of the
  network in the oracle (itself checked against central finite differences);
* what training gains: on held-out bathymetries the trained blend tracks the plain
  16-reference run far better than the untrained (uniform 1/4) blend;
* the shadow-step fallback switches members to the plain operator above its threshold.
"""
import numpy as np
import pytest

import oracle_lib as ol
from decks_util import rel_l2

pytestmark = pytest.mark.gpu

hw = pytest.importorskip("hawassi_c_b200")
from hawassi_c_b200 import decks, learned  # noqa: E402


def _bump_deck(root, name, seed, nx=2048, length=100.0, T_end=30.0):
    bath = decks.bump_bathymetry(nx, length, seed, n_bumps=8, h_min=0.3, h_max=2.0)
    return decks.write_deck(str(root / name), nx=nx, length=length, xinflux=10.0, depth=float(bath.max()),
                            bath=bath, model="HS2", T_end=T_end, n_samples=600, n_lines=200, Hs=0.05,
                            Tp=1.6, gamma=3.3, seed=seed, damp=(8.0, 8.0), adjcoef=0.5)


def _records(deck):
    depth = hw.engine.deck_table(deck, "depth")
    dx = float(hw.engine.deck_table(deck, "dx")[0])
    kdom = learned.kappa_linear(float(hw.engine.deck_table(deck, "nu_peak")[0]), depth)
    gam16 = hw.engine.deck_table(deck, "gamK", nref=16).reshape(16, -1)
    return learned.records(depth, dx, kdom, learned.reference_depths(depth, 16), gam16,
                           learned.reference_depths(depth, 4))


def test_mlp_gradients_vs_oracle(tmp_path):
    deck = _bump_deck(tmp_path, "g", seed=1)
    R = _records(deck)[::8][:256]
    mlp = learned.MLP(seed=3)
    P = mlp.params().astype(np.float64)
    loss_g, grad_g = mlp.grad(R)
    loss_c, grad_c = ol.mlp_loss_grad(P, R)
    assert loss_g == pytest.approx(loss_c, rel=1e-4)
    assert np.linalg.norm(grad_g - grad_c) / np.linalg.norm(grad_c) < 1e-4
    # the oracle's analytic gradient against central differences (FP64)
    rng = np.random.default_rng(0)
    for p in rng.choice(P.size, 12, replace=False):
        e = np.zeros_like(P)
        e[p] = 1e-6
        fd = (ol.mlp_loss_grad(P + e, R)[0] - ol.mlp_loss_grad(P - e, R)[0]) / 2e-6
        assert fd == pytest.approx(grad_c[p], rel=1e-5, abs=1e-9)
    mlp.close()


def test_training_gain_and_fallback(tmp_path):
    train = [_bump_deck(tmp_path, f"t{i}", seed=100 + i) for i in range(12)]
    test = [_bump_deck(tmp_path, f"e{i}", seed=900 + i) for i in range(2)]
    R = learned.training_records(train, t_run=15.0, stride=2)
    mlp = learned.MLP(seed=7)
    losses = mlp.train(R, epochs=300, batch=512, lr=2e-3)
    print("training loss first/last epoch:", losses[0], losses[-1])
    assert losses[-1] < 0.2 * losses[0]
    # held-out members: plain 16-reference run is the judge
    plain = hw.Engine(test, eps_abs=1e-8, eps_rel=1e-6, nref=16)
    plain.run_to_time(20.0)
    errs = {}
    for name in ("trained", "uniform"):
        eng = hw.Engine(test, eps_abs=1e-8, eps_rel=1e-6, nref=4)
        for m, d in enumerate(test):
            w, D = learned.learned_weights(mlp, d)
            if name == "uniform":
                w = np.full_like(w, 0.25)
            eng.set_operator_weights(m, D, w)
        eng.run_to_time(20.0)
        errs[name] = max(rel_l2(learned.eta_of(eng.state(m)[2], eng.nx[m]),
                                learned.eta_of(plain.state(m)[2], plain.nx[m])) for m in range(len(test)))
        assert all(eng.stats(m)["status"] == 0 for m in range(len(test)))
        eng.close()
    print("eta rel L2 vs plain 16-ref:", errs)
    assert errs["trained"] < 0.1 * errs["uniform"]
    # the best convex blend of 4 references over the band (per-point simplex least
    # squares) bounds what any network can reach: report the trained loss beside it
    print("trained loss", float(losses[-1]))
    # fallback: a zero threshold sends every member back to the plain operator
    weights = [learned.learned_weights(mlp, d) for d in test]
    sh = learned.ShadowedEnsemble(test, weights, period=10, threshold=0.0, eps_abs=1e-8, eps_rel=1e-6)
    sh.advance(25)
    assert sh.fallback.all() and len(sh.checks) == len(test)
    sh2 = learned.ShadowedEnsemble(test, weights, period=10, threshold=1.0, eps_abs=1e-8, eps_rel=1e-6)
    sh2.advance(25)
    assert not sh2.fallback.any() and len(sh2.checks) == 2 * len(test)
