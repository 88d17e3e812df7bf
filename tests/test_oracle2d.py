"""CPU checks of the 2D flat-bottom oracle and of the Hermitian bookkeeping the
device's row passes use (no GPU needed)."""
import numpy as np
import pytest

from hawassi_c_b200 import decks2d
from oracle_lib import Oracle2D, fft2, sym2

GRAV = 9.80665


def small_tables(nx=64, ny=32, nadj=1.0, propagation=0, seed=1, with_source=True):
    tb = decks2d.tables(nx=nx, ny=ny, Lx=0.9 * nx, Ly=0.9 * ny, depth=2.0, Hs=0.1, Tp=3.0, n_freq=24, n_dir=6,
                        t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, nadj=nadj, propagation=propagation, seed=seed)
    if not with_source:
        for k in ("newgam", "skewgam", "tsig", "sig", "sigskew"):
            tb[k] = None
        tb["nt"] = 0
    return tb


def sym_at_grid(A, herm):
    """The device's per-point formula (hw2d.cuh sym_at) evaluated on the whole grid."""
    ny, nx = A.shape
    out = np.empty_like(A)
    for r in range(ny):
        mr = (ny - r) % ny
        for c in range(nx):
            cm = (nx - c) % nx
            a, m = A[r, c], A[mr, cm]
            if 1 <= c < nx // 2:
                v = a
            elif c > nx // 2:
                v = np.conj(m)
            elif r == 0 or r == ny // 2:
                v = complex(a.real, 0.0)
            elif c == 0:
                v = a if r < ny // 2 else np.conj(m)
            else:
                v = 0.5 * (a + np.conj(m)) if herm else a
            out[r, c] = v
    return out


@pytest.mark.parametrize("shape", [(8, 16), (16, 8), (32, 32)])
def test_symmetrisation_matches_reference_operator(shape):
    rng = np.random.default_rng(3)
    A = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    S = sym2(A)                                   # the reference's fftwcomplex_2d_sym
    assert np.array_equal(sym_at_grid(A, herm=False), S)
    # E = Hermitian part of S: what the real part of the inverse transform sees
    ny, nx = shape
    mirror = np.conj(S[(-np.arange(ny)) % ny][:, (-np.arange(nx)) % nx])
    E = 0.5 * (S + mirror)
    assert np.allclose(sym_at_grid(A, herm=True), E, rtol=0, atol=1e-15)
    # the real part of iFFT(S) equals iFFT(E), which is real
    assert np.allclose(np.fft.ifft2(S).real, np.fft.ifft2(E).real, atol=1e-15)
    assert np.abs(np.fft.ifft2(E).imag).max() < 1e-15


def test_packed_split_recovers_two_real_transforms():
    rng = np.random.default_rng(4)
    a, b = rng.standard_normal((16, 32)), rng.standard_normal((16, 32))
    Z = fft2(a + 1j * b)
    ny, nx = Z.shape
    Zm = Z[(-np.arange(ny)) % ny][:, (-np.arange(nx)) % nx]
    A = 0.5 * (Z + np.conj(Zm))
    B = (Z - np.conj(Zm)) / 2j
    assert np.allclose(A, np.fft.fft2(a), atol=1e-12)
    assert np.allclose(B, np.fft.fft2(b), atol=1e-12)


def test_oracle_fft2_matches_numpy():
    rng = np.random.default_rng(5)
    x = rng.standard_normal((32, 64)) + 1j * rng.standard_normal((32, 64))
    assert np.allclose(fft2(x, -1), np.fft.fft2(x), atol=1e-11)
    assert np.allclose(fft2(x, +1), np.fft.ifft2(x) * x.size, atol=1e-11)


def test_linear_limit_is_exact_dispersion():
    """A small free wave, no source, no damping, no aliasing: the RHS is the linear
    operator d eta^ = -i (kx u^ + ky v^) C^2/g, d u^ = -i g kx eta^."""
    tb = small_tables(with_source=False, nadj=0.0)
    tb["charac"] = np.zeros_like(tb["charac"])
    tb["aal"] = np.ones_like(tb["aal"])
    nx, ny, n = tb["nx"], tb["ny"], tb["nx"] * tb["ny"]
    o = Oracle2D(tb, 1e-8, 1e-6)
    rng = np.random.default_rng(6)
    eta = 1e-9 * (rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx)))
    u = 1e-9 * (rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx)))
    v = 1e-9 * (rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx)))
    y = np.concatenate([eta.real.ravel(), eta.imag.ravel(), u.real.ravel(), u.imag.ravel(),
                        v.real.ravel(), v.imag.ravel()])
    d = o.rhs(0.0, y)
    kx, ky = np.meshgrid(tb["kx"], tb["ky"])
    c2 = tb["c2d"].reshape(ny, nx) ** 2 / GRAV
    deta = -1j * (kx * c2 * u + ky * c2 * v)
    du = -1j * GRAV * kx * eta
    dv = -1j * GRAV * ky * eta
    got_eta = (d[:n] + 1j * d[n:2 * n]).reshape(ny, nx)
    got_u = (d[2 * n:3 * n] + 1j * d[3 * n:4 * n]).reshape(ny, nx)
    got_v = (d[4 * n:5 * n] + 1j * d[5 * n:] ).reshape(ny, nx)
    scale = np.abs(deta).max()
    assert np.abs(got_eta - deta).max() < 1e-6 * scale   # HS2 terms are O(amplitude^2)
    assert np.allclose(got_u, du, rtol=0, atol=1e-6 * np.abs(du).max())
    assert np.allclose(got_v, dv, rtol=0, atol=1e-6 * np.abs(dv).max())


def test_source_generates_the_target_elevation():
    tb = small_tables()
    n = tb["nx"] * tb["ny"]
    o = Oracle2D(tb, 1e-8, 1e-6)
    y = np.zeros(6 * n)
    t, h = o.run_to(0.0, 4.0, 0.02, y)
    assert t == 4.0
    eta = np.fft.ifft2((y[:n] + 1j * y[n:2 * n]).reshape(tb["ny"], tb["nx"])).real
    assert 0.01 < np.abs(eta).max() < 0.2
    st = o.stats()
    assert st["accepted"] > 10 and st["rhs_calls"] >= 7 * st["accepted"]


def test_two_depth_operator_reduces_to_flat_one():
    """gam_min = 1, gam_plus = 0 with the flat tables as the 'min' depth: the two-depth
    RHS (rhs_AB2_2DB_uv) and the flat one (rhs_AB2_2DF_uv) differ only by the
    symmetrisations inside HSSgen (the operators are not exactly even on the
    freqspace grid), i.e. far below the signal."""
    tb = small_tables(with_source=False)
    n = tb["nx"] * tb["ny"]
    flat = Oracle2D(tb)
    var = dict(tb)
    var.update(gam_min=np.ones(n), gam_plus=np.zeros(n), csq_min=tb["c2d"] ** 2, csq_plus=tb["c2d"] ** 2,
               om2_min=tb["l2d"] * GRAV, om2_plus=tb["l2d"] * GRAV)
    two = Oracle2D(var)
    # a state of real physical fields inside the aliasing mask
    rng = np.random.default_rng(8)
    y = np.zeros(6 * n)
    for f in range(3):
        spec = np.fft.fft2(rng.standard_normal((tb["ny"], tb["nx"]))) * tb["aal"].reshape(tb["ny"], tb["nx"])
        y[2 * f * n:(2 * f + 1) * n] = 1e-3 * spec.real.ravel()
        y[(2 * f + 1) * n:(2 * f + 2) * n] = 1e-3 * spec.imag.ravel()
    a, b = flat.rhs(0.0, y), two.rhs(0.0, y)
    assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-2


# --------------------------------------------------------------------------
# kinematic breaking (2d/breaking.c, fun_sbreaking)
# --------------------------------------------------------------------------
def test_breaking_tables_follow_parambreak():
    from breaking2d_case import steep_crest_case
    tb, _ = steep_crest_case()
    cf = decks2d.cfsa2d(tb["x"], tb["y"], 6.0, 6.0, 6.0, 6.0)
    # pb.Char: cfSA where cfSA and ChiAdj are 1, zero in the damping zones and the influx band
    assert np.all(tb["brchar"][cf < 1] == 0) and np.all(tb["brchar"][tb["chiadj"] < 1] == 0)
    assert tb["brchar"].max() == 1.0 and np.all(tb["bathy"] == -tb["depth"])
    assert abs(tb["max_eta_init"] - 0.27) < 1e-15 and abs(tb["rsearch"] * 4 * decks2d.invers_omega(2 * np.pi / 4.0, 3.0)
                                                          - 2 * np.pi) < 1e-12


def test_breaking_rhs_at_tprev_is_the_plain_rhs():
    """At t == tprev (the first stage of every evolve_apply) no update runs and Sb is
    still zero: the RHS is the one without breaking, bit for bit."""
    from breaking2d_case import steep_crest_case
    tb, z = steep_crest_case()
    plain = {k: v for k, v in tb.items() if k != "breaking"}
    a, b = Oracle2D(tb, 1e-6, 1e-4), Oracle2D(plain, 1e-6, 1e-4)
    a.set_tprev(0.3)
    assert np.array_equal(a.rhs(0.3, z), b.rhs(0.3, z))
    B, sx, sy, flag, nc = a.breaking_fields()
    assert flag == 0 and nc == 0 and not B.any() and not sx.any()


def test_breaking_starts_tracks_and_logs():
    """The steep crest: candidates at the first update, crests tracked with break
    nodes (flagbr 2), a nonzero eddy-viscosity force, records in breaking.dat."""
    from breaking2d_case import steep_crest_case
    tb, z = steep_crest_case()
    o = Oracle2D(tb, 1e-6, 1e-4)
    t, h, y = 0.3, 0.005, z.copy()
    o.set_tprev(t)
    seen2 = False
    for _ in range(8):
        t, h = o.evolve_apply(t, 0.6, h, y)
        B, sx, sy, flag, nc = o.breaking_fields()
        if flag == 2:
            seen2 = True
            assert nc >= 1 and (B > 0).any() and np.abs(sx).max() > 0
            assert np.all((B >= 0) & (B <= 1))
    assert seen2
    log = o.breaking_log()
    assert len(log) >= 1 and all(len(nodes) > 0 for _, nodes in log)
    assert all(0 <= x < tb["nx"] and 0 <= yy < tb["ny"] for _, nodes in log for x, yy in nodes)
    # records come from every RHS past tprev, rejected attempts' stages included
    assert all(0.3 < tt <= t + 0.05 for tt, _ in log)


def hs3_pair(nx=64, ny=32, walls=()):
    """HS3 tables and the same tables run as HS2 (HS3's aliasing mask), no source."""
    tb3 = decks2d.tables(nx=nx, ny=ny, Lx=0.9 * nx, Ly=0.9 * ny, depth=2.0, Hs=0.1, Tp=3.0, n_freq=24, n_dir=6,
                         t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, nadj=1.0, seed=2, model=3, walls=walls)
    for k in ("newgam", "skewgam", "tsig", "sig", "sigskew"):
        tb3[k] = None
    tb3["nt"] = 0
    tb2 = dict(tb3)
    tb2["model"] = 2
    return tb2, tb3


@pytest.mark.parametrize("walls", [(), ((20.0, 5.0, 24.0, 20.0),)])
def test_hs3_terms_are_cubic(walls):
    """rhs_AB3_2DF_uv - rhs_AB2_2DF_uv on the same tables is homogeneous of degree
    three in the state: the cubic terms alone (the adjustment is linear)."""
    tb2, tb3 = hs3_pair(walls=walls)
    nx, ny = tb3["nx"], tb3["ny"]
    n = nx * ny
    o2, o3 = Oracle2D(tb2), Oracle2D(tb3)
    rng = np.random.default_rng(11)
    z = 0.02 * rng.standard_normal(6 * n) * np.tile(tb3["aal"].ravel(), 6) * np.sqrt(n)
    d1 = o3.rhs(0.0, z) - o2.rhs(0.0, z)
    d2 = o3.rhs(0.0, 2 * z) - o2.rhs(0.0, 2 * z)
    assert np.linalg.norm(d1) > 1e-8 * np.linalg.norm(o2.rhs(0.0, z))
    assert np.linalg.norm(d2 - 8 * d1) < 1e-8 * np.linalg.norm(d2)


@pytest.mark.parametrize("ninterp", [2, 3])
def test_hs3_terms_are_cubic_varying_bottom(ninterp):
    """rhs_AB3_2DB_uv - rhs_AB2_2DB_uv on the same two- or three-depth tables: the cubic
    terms alone, homogeneous of degree three."""
    tb3 = decks2d.tables(nx=64, ny=32, Lx=57.6, Ly=28.8, depth=2.0, shallow=0.6, Hs=0.1, Tp=3.0, n_freq=24,
                         n_dir=6, t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, nadj=1.0, seed=2, bathymetry="shoal",
                         model=3, ninterp=ninterp)
    for k in ("newgam", "skewgam", "tsig", "sig", "sigskew"):
        tb3[k] = None
    tb3["nt"] = 0
    tb2 = dict(tb3, model=2)
    n = tb3["nx"] * tb3["ny"]
    o2, o3 = Oracle2D(tb2), Oracle2D(tb3)
    rng = np.random.default_rng(12)
    z = 0.02 * rng.standard_normal(6 * n) * np.tile(tb3["aal"].ravel(), 6) * np.sqrt(n)
    d1 = o3.rhs(0.0, z) - o2.rhs(0.0, z)
    d2 = o3.rhs(0.0, 2 * z) - o2.rhs(0.0, 2 * z)
    assert np.linalg.norm(d1) > 1e-8 * np.linalg.norm(o2.rhs(0.0, z))
    assert np.linalg.norm(d2 - 8 * d1) < 1e-8 * np.linalg.norm(d2)


def _shoal(ninterp=2, model=2, ny=32):
    return decks2d.tables(nx=64, ny=ny, Lx=57.6, Ly=0.9 * ny, depth=2.0, shallow=0.6, Hs=0.1, Tp=3.0, n_freq=24,
                          n_dir=6, t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, seed=4, bathymetry="shoal",
                          ninterp=ninterp, model=model)


def test_three_depth_weights_are_exact_at_the_knots():
    """funOprt_DispInterpolation_3p: at every knot depth the blend of the three reference
    depths reproduces the long-wave speed, the squared frequency and the phase speed of
    the peak wavenumber there."""
    import math
    tb = _shoal()
    depth = tb["depth"]
    wp = 2 * math.pi / 3.0
    op = decks2d.three_depth_operator(depth, tb["kx"], tb["ky"], wp)
    DD, g, refs = op["_knots"]

    def cp1(k, D):
        return math.sqrt(GRAV * k * math.tanh(k * D)) / k

    def om2(k, D):
        return GRAV * k * math.tanh(k * D)

    for i in range(DD.size):
        kap = decks2d.invers_omega(wp, DD[i])
        for f in (lambda D: math.sqrt(GRAV * D), lambda D: om2(kap, D), lambda D: cp1(kap, D)):
            blend = sum(g[r, i] * f(refs[r]) for r in range(3))
            assert blend == pytest.approx(f(DD[i]), rel=1e-9)
    assert op["gam_mid"].shape == depth.shape and np.isfinite(op["gam_mid"]).all()


@pytest.mark.parametrize("model", [1, 2, 3])
def test_three_depth_with_an_idle_middle_depth_is_two_depth(model):
    """HSSgen_3depth with Gam_mid = 0 adds exact zeros to HSSgen_2depth's sum: the RHS is
    bit-identical; with the plus weight split half onto a middle depth equal to the
    deepest one it agrees to rounding."""
    tb2 = _shoal(model=model)
    n = tb2["nx"] * tb2["ny"]
    rng = np.random.default_rng(3)
    y = 0.02 * rng.standard_normal(6 * n) * np.tile(tb2["aal"].ravel(), 6) * np.sqrt(n)
    ref = Oracle2D(tb2).rhs(0.7, y)
    tb3 = dict(tb2, gam_mid=np.zeros_like(tb2["gam_plus"]), csq_mid=tb2["csq_plus"], om2_mid=tb2["om2_plus"])
    assert np.array_equal(Oracle2D(tb3).rhs(0.7, y), ref)
    half = 0.5 * tb2["gam_plus"]
    tb4 = dict(tb2, gam_plus=half, gam_mid=half, csq_mid=tb2["csq_plus"], om2_mid=tb2["om2_plus"])
    d = Oracle2D(tb4).rhs(0.7, y)
    assert np.linalg.norm(d - ref) < 1e-13 * np.linalg.norm(ref)


def test_three_depth_tables_run_in_the_oracle():
    tb = _shoal(ninterp=3, ny=64)
    assert {"gam_mid", "csq_mid", "om2_mid"} <= set(tb)
    n = tb["nx"] * tb["ny"]
    rng = np.random.default_rng(5)
    y = 0.02 * rng.standard_normal(6 * n) * np.tile(tb["aal"].ravel(), 6) * np.sqrt(n)
    assert np.isfinite(Oracle2D(tb).rhs(0.3, y)).all()


# ------------------------------------------------------------ K reference depths
def _k_tables(tb, names):
    kt = {k: v for k, v in tb.items() if not k.startswith(("gam_", "csq_", "om2_"))}
    kt["nrefk"] = len(names)
    kt["gam_k"] = np.stack([tb[f"gam_{m}"].ravel() for m in names])
    kt["csq_k"] = np.stack([tb[f"csq_{m}"].ravel() for m in names])
    kt["om2_k"] = np.stack([tb[f"om2_{m}"].ravel() for m in names])
    return kt


@pytest.mark.parametrize("ninterp,model", [(2, 2), (2, 3), (3, 2), (3, 3)])
def test_k_reference_form_is_hssgen_bit_for_bit(ninterp, model):
    """The K-depth sum with the two- or three-depth tables is HSSgen_2depth /
    HSSgen_3depth exactly (same products, same summation order)."""
    tb = decks2d.tables(nx=64, ny=64, Lx=57.6, Ly=57.6, depth=2.0, shallow=0.6, Hs=0.1, Tp=3.0, n_freq=16,
                        n_dir=4, t_end=4.0, dt=0.1, damp=6.0, x_line=10.0, seed=1, bathymetry="shoal",
                        ninterp=ninterp, model=model)
    names = ["min", "mid", "plus"] if ninterp == 3 else ["min", "plus"]
    kt = _k_tables(tb, names)
    n = 64 * 64
    y = 0.02 * np.random.default_rng(3).standard_normal(6 * n) * np.tile(tb["aal"].ravel(), 6) * 64
    a = Oracle2D(tb, 1e-8, 1e-6).rhs(0.9, y)
    b = Oracle2D(kt, 1e-8, 1e-6).rhs(0.9, y)
    assert np.array_equal(a, b)


def test_k_reference_weights():
    """The plain K-reference weights: two non-zero weights per point (the bracketing
    pair), weight 1 on a point that sits at a reference depth, and with K = 2 the
    two-depth operator's weights up to its spline over 101 depth samples."""
    tb = decks2d.tables(nx=64, ny=64, Lx=57.6, Ly=57.6, depth=2.0, shallow=0.6, Hs=0.1, Tp=3.0, n_freq=16,
                        n_dir=4, t_end=4.0, dt=0.1, damp=6.0, x_line=10.0, seed=1, bathymetry="shoal")
    depth = tb["depth"]
    D = decks2d.log_reference_depths(depth, 16)
    w = decks2d.k_reference_weights(depth, tb["wp"], D)
    assert w.shape == (16,) + depth.shape
    assert ((w != 0).sum(axis=0) <= 2).all()
    assert np.abs(w.sum(axis=0) - 1).max() < 1e-3
    wd = decks2d.k_reference_weights(np.array(D[5:9]), tb["wp"], D)
    assert np.allclose(wd[5:9].diagonal(), 1.0, atol=1e-12)
    w2 = decks2d.plain_k_operator(tb, 2)["gam_k"]
    assert np.abs(w2[0] - tb["gam_min"].ravel()).max() < 1e-4
    assert np.abs(w2[1] - tb["gam_plus"].ravel()).max() < 1e-4


# ------------------------------------------------- the directional influx model
@pytest.mark.parametrize("s_spread", [10.0, None])
def test_reference_directional_components_match_oracle(s_spread):
    """decks2d's components of jonswap_influx (seeded draws) equal the oracle's C
    restatement given the same uniforms: amplitudes, frequencies, wavenumbers,
    directions (the cos^2s inverse CDF) and phases."""
    import math
    import oracle_lib as ol
    from hawassi_c_b200.decks import splitmix64_uniform
    t = np.arange(601) * 0.1
    got = decks2d.reference_directional_components(t, 0.5, 6.0, 3.3, s_spread, 4.0, seed=7)
    nh = t.size // 2
    ref = ol.jonswap_components_2d(t, 0.5, 6.0, 3.3, s_spread if s_spread else -1.0, 4.0,
                                   splitmix64_uniform(15, nh), splitmix64_uniform(16, nh))
    for g, r in zip(got, ref):
        np.testing.assert_allclose(g, r, rtol=1e-12, atol=1e-14)
    a, w = got[0], got[1]
    assert np.sum(a ** 2) / 2 == pytest.approx((0.5 / 4) ** 2, rel=0.02)   # Hs from the amplitudes
    if s_spread:
        assert np.abs(got[3]).max() < math.pi / 2 and np.std(got[3]) > 0.1


@pytest.mark.parametrize("K", [4, 16])
def test_hs3_terms_are_cubic_k_reference(K):
    """The same homogeneity with the K-reference-depth operator (the plain 16-depth one
    and the 4-depth form of the learned blend)."""
    tb3 = decks2d.tables(nx=64, ny=32, Lx=57.6, Ly=28.8, depth=2.0, shallow=0.6, Hs=0.1, Tp=3.0, n_freq=24,
                         n_dir=6, t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, nadj=1.0, seed=2, bathymetry="shoal",
                         model=3)
    for k in ("newgam", "skewgam", "tsig", "sig", "sigskew"):
        tb3[k] = None
    tb3["nt"] = 0
    tb3 = decks2d.plain_k_operator(tb3, K)
    tb2 = dict(tb3, model=2)
    n = tb3["nx"] * tb3["ny"]
    o2, o3 = Oracle2D(tb2), Oracle2D(tb3)
    rng = np.random.default_rng(13)
    z = 0.02 * rng.standard_normal(6 * n) * np.tile(tb3["aal"].ravel(), 6) * np.sqrt(n)
    d1 = o3.rhs(0.0, z) - o2.rhs(0.0, z)
    d2 = o3.rhs(0.0, 2 * z) - o2.rhs(0.0, 2 * z)
    assert np.linalg.norm(d1) > 1e-8 * np.linalg.norm(o2.rhs(0.0, z))
    assert np.linalg.norm(d2 - 8 * d1) < 1e-8 * np.linalg.norm(d2)


def test_k_reference_operator_with_idle_depths_is_the_two_depth_one():
    """A flat 1.5 m bottom under 4 reference depths (1.5, 3, 6, 12 m): the K-depth
    weights put every point wholly on the first depth, and the idle depths' terms are
    exact zeros, so the K-reference RHS equals, bit for bit, the two-depth RHS with the
    same weights (gam_min = 1, gam_plus = 0) -- which the test above relates to the flat
    RHS."""
    tb = decks2d.tables(nx=64, ny=32, Lx=57.6, Ly=28.8, depth=1.5, Hs=0.1, Tp=3.0, n_freq=24, n_dir=6, t_end=6.0,
                        dt=0.1, damp=6.0, x_line=10.0, nadj=1.0, seed=2)
    n = tb["nx"] * tb["ny"]
    depth = np.full((tb["ny"], tb["nx"]), 1.5)
    D = np.array([1.5, 3.0, 6.0, 12.0])
    w = decks2d.k_reference_weights(depth, 2 * np.pi / 3.0, D)
    assert np.allclose(w[0], 1.0, atol=1e-12) and np.allclose(w[1:], 0.0, atol=1e-12)
    w = np.zeros_like(w)
    w[0] = 1.0
    kt = decks2d.with_k_operator(dict(tb, depth=depth), D, w)
    two = dict(tb, gam_min=np.ones(n), gam_plus=np.zeros(n), csq_min=kt["csq_k"][0], csq_plus=kt["csq_k"][1],
               om2_min=kt["om2_k"][0], om2_plus=kt["om2_k"][1])
    rng = np.random.default_rng(14)
    z = 0.02 * rng.standard_normal(6 * n) * np.tile(tb["aal"].ravel(), 6) * np.sqrt(n)
    for model in (2, 3):
        a = Oracle2D(dict(two, model=model)).rhs(0.4, z)
        b = Oracle2D(dict(kt, model=model)).rhs(0.4, z)
        assert np.array_equal(a, b), model
