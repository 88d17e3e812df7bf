"""Host-side pieces of the learned operator's 2D variant (no GPU): the 2D depth
features, the K-reference tables dict and the domain-filling sea state the
comparison starts from."""
import math

import numpy as np

from hawassi_c_b200 import decks2d, learned


def _shoal(n=64):
    return decks2d.tables(nx=n, ny=n, Lx=0.9 * n, Ly=0.9 * n, depth=2.0, shallow=0.6, Hs=0.1, Tp=3.0, n_freq=16,
                          n_dir=4, t_end=4.0, dt=0.1, damp=6.0, x_line=10.0, seed=1, bathymetry="shoal")


def test_features2d_layout_and_flat_limit():
    tb = _shoal()
    depth = tb["depth"]
    kdom = learned.kappa_linear(float(tb["wp"]), depth)
    f = learned.features2d(depth, float(tb["dx"]), float(tb["dy"]), kdom)
    assert f.shape == (depth.size, 5) and f.dtype == np.float32 and np.isfinite(f).all()
    # the depth itself sits on the log scale of the 4 reference depths: -1.5 .. 1.5
    assert f[:, 0].min() == np.float32(-1.5) and abs(float(f[:, 0].max()) - 1.5) < 1e-5
    # on a nearly flat bottom every point gets nearly the same dominant-band feature
    flat = np.full((32, 32), 1.3) * np.linspace(1.0, 1.0001, 32)[None, :]
    g = learned.features2d(flat, 0.5, 0.5, learned.kappa_linear(2.0, flat))
    assert np.ptp(g[:, 4]) < 1e-3


def test_k_operator_tables_replace_the_two_depth_ones():
    tb = _shoal()
    k16 = decks2d.plain_k_operator(tb, 16)
    n = tb["nx"] * tb["ny"]
    assert k16["nrefk"] == 16 and k16["gam_k"].shape == (16, n)
    assert k16["csq_k"].shape == (16, n) and k16["om2_k"].shape == (16, n)
    assert not any(k.startswith(("gam_min", "gam_plus", "csq_min", "om2_min")) for k in k16)
    D = k16["ref_depths"]
    assert D[0] == tb["depth"].min() and D[-1] == tb["depth"].max() and np.all(np.diff(D) > 0)


def test_wave_field_fills_the_domain_with_the_asked_height():
    tb = _shoal(128)
    y = learned.wave_field_2d(tb, seed=4, hs_frac=0.5)
    n = tb["nx"] * tb["ny"]
    eta = np.fft.ifft2((y[:n] + 1j * y[n:2 * n]).reshape(tb["ny"], tb["nx"])).real
    assert abs(4 * eta.std() - 0.5 * tb["hs"]) < 0.1 * 0.5 * tb["hs"]
    assert np.all(y[2 * n:] == 0)                       # u = v = 0
    # both halves of the domain carry waves (not a wave train from one line)
    left, right = eta[:, : tb["nx"] // 2], eta[:, tb["nx"] // 2:]
    assert left.std() > 0.3 * right.std() and right.std() > 0.3 * left.std()
    assert math.isfinite(float(eta.max()))
