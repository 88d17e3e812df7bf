"""The general 2D path on the varying bottom (hw2d_gen.cuh) against the 2D oracle.

It runs rhs_AB1/AB2/AB3_2DB_uv as the reference's sequence of whole-field
operations, for what the fused passes do not cover: three reference depths
(HSSgen_3depth) under HS1, HS2 and HS3, and HS3 with two reference depths.  The
bar is the fused paths': one RHS 1e-11 relative L2 (walls, source, breaking),
evolve steps with the same step sizes and counts, state 1e-9, identical
breaking records.  Also here: the fused two-depth path at the configuration's
own grid, 1024 x 1024, with a harbour wall and breaking."""
import numpy as np
import pytest

from breaking2d_case import steep_crest_case
from hawassi_c_b200 import decks2d
from hawassi_c_b200.engine2d import Engine2D
from oracle_lib import Oracle2D

pytestmark = pytest.mark.gpu


def shoal(nx, ny, ninterp=3, model=2, walls=(), seed=4):
    return decks2d.tables(nx=nx, ny=ny, Lx=0.9 * nx, Ly=0.9 * ny, depth=2.0, shallow=0.6, Hs=0.1, Tp=3.0,
                          n_freq=24, n_dir=6, t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, seed=seed,
                          bathymetry="shoal", ninterp=ninterp, model=model, walls=walls)


def band_limited_state(tb, amp, seed):
    rng = np.random.default_rng(seed)
    n = tb["nx"] * tb["ny"]
    return amp * rng.standard_normal(6 * n) * np.tile(tb["aal"].ravel(), 6) * np.sqrt(n)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("nx,ny,ninterp,model", [
    (64, 64, 3, 2), (128, 64, 3, 1), (64, 128, 3, 3), (64, 64, 2, 3), (128, 128, 3, 2), (256, 128, 2, 3),
])
def test_general_rhs_parity(nx, ny, ninterp, model):
    tb = shoal(nx, ny, ninterp=ninterp, model=model)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    for seed, t in ((1, 0.7), (2, 3.3)):
        y = band_limited_state(tb, 0.02, seed)
        assert rel(eng.rhs(t, y), ora.rhs(t, y)) < 1e-11


@pytest.mark.parametrize("model", [2, 3])
def test_general_rhs_parity_walls_unfiltered(model):
    """A harbour wall (wallchar in the products), every wavenumber excited."""
    tb = shoal(128, 64, ninterp=3, model=model, walls=((30.0, 20.0, 33.0, 45.0),))
    eng, ora = Engine2D(tb), Oracle2D(tb)
    rng = np.random.default_rng(9)
    y = 0.01 * rng.standard_normal(6 * tb["nx"] * tb["ny"]) * 90
    assert rel(eng.rhs(1.0, y), ora.rhs(1.0, y)) < 1e-11


@pytest.mark.parametrize("ninterp,model", [(3, 2), (2, 3)])
def test_general_run_parity(ninterp, model):
    """The graph-replayed device loop to t = 1.5 s from rest, driven by the line source."""
    tb = shoal(64, 64, ninterp=ninterp, model=model)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    n = tb["nx"] * tb["ny"]
    h0 = 0.02
    eng.set_state(0.0, h0, np.zeros(6 * n))
    y = np.zeros(6 * n)
    t, h = ora.run_to(0.0, 1.5, h0, y)
    eng.run_to_time(1.5)
    te, he, ye = eng.state()
    assert abs(te - t) < 1e-12 and abs(he - h) <= 1e-6 * abs(h)
    so, se = ora.stats(), eng.stats()
    assert (se["accepted"], se["rejected"]) == (so["accepted"], so["rejected"])
    assert np.abs(y).max() > 0 and rel(ye, y) < 1e-9


def test_general_breaking_parity():
    """Kinematic breaking with three reference depths: the breaking kernels after the
    general path's assembly, eight evolve_apply calls in step."""
    tb, z = steep_crest_case(64, 64, ninterp=3)
    eng, ora = Engine2D(tb, 1e-6, 1e-4), Oracle2D(tb, 1e-6, 1e-4)
    t0, h0 = 0.3, 0.005
    eng.set_state(t0, h0, z)
    ora.set_tprev(t0)
    ya, yb = z.copy(), z.copy()
    ta, ha, tb_, hb = t0, h0, t0, h0
    for _ in range(8):
        ta, ha = ora.evolve_apply(ta, 0.6, ha, ya)
        tb_, hb = eng.evolve_apply(tb_, 0.6, hb, yb)
        assert abs(ta - tb_) < 1e-11 and abs(ha - hb) <= 1e-6 * abs(ha)
        assert rel(yb, ya) < 1e-9
        assert eng.stats()["accepted"] == ora.stats()["accepted"]
        assert eng.stats()["rejected"] == ora.stats()["rejected"]
    la, lb = ora.breaking_log(), eng.breaking_log()
    assert len(la) > 0 and len(la) == len(lb)
    for (t1, n1), (t2, n2) in zip(lb, la):
        assert abs(t1 - t2) <= 1e-12 * max(1.0, abs(t2)) and n1 == n2


def test_rhs_parity_1024_two_depth_wall_breaking():
    """The fused two-depth path at 1024 x 1024 (the 2D configuration's grid), with a
    harbour wall and the breaking tables, one RHS past tprev, against the oracle."""
    tb, z = steep_crest_case(1024, 1024, x_crest=500.0, walls=((600.0, 300.0, 606.0, 700.0),))
    eng, ora = Engine2D(tb, 1e-6, 1e-4), Oracle2D(tb, 1e-6, 1e-4)
    eng.set_state(0.3, 0.005, z)
    ora.set_tprev(0.3)
    t = 0.304
    assert rel(eng.rhs(t, z), ora.rhs(t, z)) < 1e-11
    Be, _, _, fe, ne = eng.breaking_fields()
    Bo, _, _, fo, no = ora.breaking_fields()
    assert (fe, ne) == (fo, no) and np.array_equal(Be > 0, Bo > 0)


# ------------------------------------------------ K reference depths (plain and learned)
@pytest.mark.parametrize("K,model", [(4, 2), (16, 2), (4, 3), (16, 1)])
def test_k_reference_rhs_parity(K, model):
    """The K-reference operator (the plain 16-reference one and the 4-depth form the
    learned blend uses) on the general path: one RHS 1e-11 against the oracle's
    K-depth HSSgen sum."""
    tb = decks2d.plain_k_operator(shoal(64, 64, ninterp=2, model=model), K)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    for seed, t in ((1, 0.7), (2, 3.3)):
        y = band_limited_state(tb, 0.02, seed)
        assert rel(eng.rhs(t, y), ora.rhs(t, y)) < 1e-11


def test_k_reference_run_parity():
    """The graph-replayed loop with 16 reference depths to t = 1.5 s from rest: the
    same step counts, state 1e-9."""
    tb = decks2d.plain_k_operator(shoal(64, 64, ninterp=2), 16)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    n = tb["nx"] * tb["ny"]
    h0 = 0.02
    eng.set_state(0.0, h0, np.zeros(6 * n))
    y = np.zeros(6 * n)
    t, h = ora.run_to(0.0, 1.5, h0, y)
    eng.run_to_time(1.5)
    te, he, ye = eng.state()
    assert abs(te - t) < 1e-12 and abs(he - h) <= 1e-6 * abs(h)
    so, se = ora.stats(), eng.stats()
    assert (se["accepted"], se["rejected"]) == (so["accepted"], so["rejected"])
    assert np.abs(y).max() > 0 and rel(ye, y) < 1e-9


def test_learned_operator_2d_gain():
    """The learned K = 4 blend on a 2D bottom (the committed network, 2D features):
    against the plain 16-reference run its eta error is well below that of uniform
    weights over the same 4 depths, the method without the network."""
    from hawassi_c_b200 import learned
    mlp = learned.load_mlp()
    assert mlp is not None
    tb = decks2d.tables(nx=128, ny=128, Lx=115.2, Ly=115.2, depth=2.0, shallow=0.3, Hs=0.1, Tp=2.5, n_freq=24,
                        n_dir=6, t_end=8.0, dt=0.1, damp=8.0, x_line=12.0, seed=5, bathymetry="shoal")
    plain = decks2d.plain_k_operator(tb, 16)
    lrn = learned.learned_tables2d(mlp, tb)
    D4 = lrn["ref_depths"]
    uni = decks2d.with_k_operator(tb, D4, np.full((4,) + tb["depth"].shape, 0.25))
    n = tb["nx"] * tb["ny"]
    etas = {}
    for name, t in (("plain", plain), ("learned", lrn), ("uniform", uni)):
        e = Engine2D(t, 1e-8, 1e-6)
        e.set_state(0.0, 0.02, np.zeros(6 * n))
        e.run_to_time(6.0)
        etas[name] = e.fields()[0]
        e.close()
    err = {k: rel(etas[k], etas["plain"]) for k in ("learned", "uniform")}
    assert np.abs(etas["plain"]).max() > 0
    assert err["learned"] < 0.2 * err["uniform"], err
