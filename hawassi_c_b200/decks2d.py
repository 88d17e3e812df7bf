"""Operator tables of the HAWASSI 2D flat-bottom RHS for seeded synthetic decks.

The 2D RHS (2d/fun_odesolver.c:4404-4540) reads tables that the reference's
set-up builds: the wavenumber grids (freqspace, 2d/functions.c:1810-1832), the
exact-dispersion operators C2d and L2d (fun_operator_setup, :1514-1523), the
aliasing mask (fun_aal2D, :1834-1880), the damping characteristic (fun_fbdy2D /
fun_cfSA2D, :1958-2132), the nonlinear adjustment ChiAdj (fun_calcseacharacteristic
with cfv, :787-793, :905-921), the area-source kernels newGam / SkewGam
(fun_area_generation, vertical influx line, :2991-3085) and one influx signal
per row (Spline_Signal / Spline_SkewSignal, :3241-3250).  This module restates
those constructions in numpy for a flat bottom, no wall, no coupling and a
vertical influx line spanning the domain, and synthesises the line signals from
a seeded directional JONSWAP spectrum (cos^2s spreading) on the (ky, omega) grid.

`tables()` returns a dict with the arrays the engine's `hw2d_tables` takes.
"""
from __future__ import annotations

import math

import numpy as np

GRAV = 9.80665   # 2d/var_initialization.h:246


def freqspace(length: float, n: int) -> np.ndarray:
    """2d/functions.c:1810-1832 (its quirks included: spacing 2 pi (N-2)/(len (N-1))
    for even N, and k[0] = 1e-10)."""
    dk = 2 * math.pi / length
    fmin = -0.5 * 2 * math.pi / (length / (n - 1))
    fmax = -fmin - dk if n % 2 == 0 else -fmin
    d = (fmax - fmin) / (n - 1)
    out = np.empty(n)
    for i in range(n // 2):
        out[i] = fmin + (n // 2 + i) * d
    for ni, i in enumerate(range(n // 2, n)):
        out[i] = fmin + ni * d
    out[0] = 1e-10
    return out


def aal2d(kx: np.ndarray, ky: np.ndarray, cutfrac: int) -> np.ndarray:
    """fun_aal2D (2d/functions.c:1834-1880)."""
    nx, ny = kx.size, ky.size
    idx = max(int(math.floor(nx / cutfrac)) - 1, 0)
    idy = max(int(math.floor(ny / cutfrac)) - 1, 0)
    kxmax, kymax = abs(kx[idx]), abs(ky[idy])
    KK = np.sqrt(kx[None, :] ** 2 + ky[:, None] ** 2)
    if idx > 0 and idy > 0:
        kmax = math.sqrt(kxmax ** 2 + kymax ** 2)
        return np.where(np.abs(KK) > kmax, 0.0, 1.0)
    alx = np.where(np.abs(kx) > kxmax, 0.0, 1.0)
    aly = np.where(np.abs(ky) > kymax, 0.0, 1.0)
    return aly[:, None] * alx[None, :]


def _closest(a: np.ndarray, ref: float) -> int:
    """fun_closest (2d/functions1.c:786-799): first index of the minimum distance."""
    return int(np.argmin(np.abs(ref - a)))


def _sign(v):
    return np.where(np.asarray(v) < 0, -1.0, 1.0)


def cfsa2d(x, y, Lleft, Lright, Lbottom, Ltop) -> np.ndarray:
    """fun_cfSA2D (2d/functions.c:2084-2132)."""
    nx, ny = x.size, y.size
    ixl = _closest(x, x[0] + Lleft)
    ixr = _closest(x, x[nx - 1] - Lright)
    iyb = _closest(y, y[0] + Lbottom)
    iyt = _closest(y, y[ny - 1] - Ltop)
    hxl = (x - x[0] >= 0).astype(float)
    hxr = (x - x[ixr] >= 0).astype(float)
    hyb = (y - y[0] >= 0).astype(float)
    hyt = (y - y[iyt] >= 0).astype(float)
    with np.errstate(divide="ignore", invalid="ignore"):
        A = _sign(x - x[ixl])
        B = (1 - np.cos((x - x[0]) * math.pi / Lleft)) / 2 if Lleft else np.zeros(nx)
        cfxl = hxl * np.maximum(A, B)
        C = _sign(x - x[nx - 1])
        D = (1 - np.cos((x - x[ixr]) * math.pi / Lright)) / 2 if Lright else np.zeros(nx)
        cfxr = hxr * np.maximum(C, D)
        if Lleft == 0:
            cfxl = np.ones(nx)
        if Lright == 0:
            cfxr = np.zeros(nx)
        E = _sign(y - y[iyb])
        F = (1 - np.cos((y - y[0]) * math.pi / Lbottom)) / 2 if Lbottom else np.zeros(ny)
        cfyb = hyb * np.maximum(E, F)
        G = _sign(y - y[ny - 1])
        H = (1 - np.cos((y - y[iyt]) * math.pi / Ltop)) / 2 if Ltop else np.zeros(ny)
        cfyt = hyt * np.maximum(G, H)
        if Lbottom == 0:
            cfyb = np.ones(ny)
        if Ltop == 0:
            cfyt = np.zeros(ny)
    return (cfyb - cfyt)[:, None] * (cfxl - cfxr)[None, :]


def cutoff(refl, model=2):
    """fun_cutoff (2d/functions.c:225-258), with the reference's operator precedence."""
    a, b, c = (0.8086, 0.2413, 0.0044) if model == 1 else (0.7289, 0.3229, -0.00058)
    if refl == 1:
        return 1.0
    if refl == 0:
        return 0.0
    return -b + math.sqrt(b ** 2 - 4 * a * (c - refl)) / (2 * a)


def _heav_band(v, lo, hi):
    """fun_Heav2d along one axis: 1 for lo <= v < hi (the side clearances 0 keep
    that side open)."""
    hb = np.ones(v.size) if lo - v[0] == 0 else (v - lo >= 0).astype(float)
    ht = np.zeros(v.size) if v[-1] - hi == 0 else (v - hi >= 0).astype(float)
    return hb * (1 - ht)


def wallchar2d(x, y, walls, refl, model=2):
    """fun_wallchar (2d/functions.c:260-390) for rectangular walls (x0, y0, x1, y1):
    wallchar = 1 - cutoff(refl) inside any wall, 1 elsewhere; cfSAwall = 0 inside the
    first wall (direct damping), 1 elsewhere."""
    heav = np.ones((y.size, x.size))
    for (x0, y0, x1, y1) in walls:
        heav *= 1 - _heav_band(y, y0, y1)[:, None] * _heav_band(x, x0, x1)[None, :]
    wc = np.where(heav == 0, 1 - cutoff(refl, model), 1.0)
    dx, dy = x[1] - x[0], y[1] - y[0]
    cfw = np.ones((y.size, x.size))
    if walls:
        x0, y0, x1, y1 = walls[0]
        i0, i1 = int(round((y0 - y[0]) / dy)), int(round((y1 - y[0]) / dy))
        j0, j1 = int(round((x0 - x[0]) / dx)), int(round((x1 - x[0]) / dx))
        cfw[i0:i1 + 1, j0:j1 + 1] = 0.0
    return wc, cfw


def fbdy2d(x, y, Lleft, Lright, Lbottom, Ltop, cfsa_wall=None, model=2) -> np.ndarray:
    """fun_fbdy2D (2d/functions.c:1958-2082), no coupling: the zone length L of the
    last matching side (7 where it is 0) scales (1 - cfSA)/(0.9 L); with walls cfSA
    is min(cfSA, cfSAwall) and the whole field is ten times stronger (not HS1)."""
    nx, ny = x.size, y.size
    cf = cfsa2d(x, y, Lleft, Lright, Lbottom, Ltop)
    if cfsa_wall is not None:
        cf = np.minimum(cf, cfsa_wall)
    ixl = _closest(x, x[0] + Lleft)
    ixr = _closest(x, x[nx - 1] - Lright)
    iyb = _closest(y, y[0] + Lbottom)
    iyt = _closest(y, y[ny - 1] - Ltop)
    out = np.empty((ny, nx))
    L = 7.0
    for i in range(ny):
        for j in range(nx):
            if j <= ixl:
                L = Lleft
            if j >= ixr:
                L = Lright
            if i < iyb and ixl < j < ixr:
                L = Lbottom
            if i > iyt and ixl < j < ixr:
                L = Ltop
            if L == 0:
                L = 7.0
            out[i, j] = (1 - cf[i, j]) / (0.9 * L)
    if cfsa_wall is not None and model != 1:
        out = 10 * out
    return out


def exact_cp(kx, ky, depth, ux=0.0, uy=0.0):
    """fun_exact_Cp_val (2d/functions.c:101-112)."""
    K = np.sqrt(kx ** 2 + ky ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        c = np.sqrt(GRAV * np.tanh(K * depth) / K) + (kx * ux + ky * uy) / K
    return np.where(K == 0, math.sqrt(GRAV * depth), c)


def exact_disp(kx, ky, depth, mdir=0.0, ux=0.0, uy=0.0):
    """fun_exact_disp_val (2d/functions.c:114-120)."""
    s = _sign(kx * math.cos(mdir) + ky * math.sin(mdir))
    K = np.sqrt(kx ** 2 + ky ** 2)
    return s * np.sqrt(GRAV * K * np.tanh(K * depth)) + kx * ux + ky * uy


def exact_ug(k, d, U=0.0):
    """fun_exact_Ug_val (2d/functions.c:82-92)."""
    k = np.asarray(k, dtype=float)
    with np.errstate(divide="ignore", invalid="ignore"):
        th = np.tanh(d * k)
        ug = _sign(k) * math.sqrt(GRAV) / 2 / np.sqrt(k * th) * (th + k * (1 - th ** 2) * d) + U
    return np.where(k == 0, math.sqrt(GRAV * d) + U, ug)


def invers_omega(w: float, depth: float) -> float:
    """Root k of w^2 = g k tanh(k depth) (Newton, as invers_omega, 2d/functions1.c:997)."""
    k = w * w / GRAV
    for _ in range(200):
        f = GRAV * k * math.tanh(k * depth) - w * w
        df = GRAV * math.tanh(k * depth) + GRAV * k * depth / math.cosh(k * depth) ** 2
        dk = f / df
        k -= dk
        if abs(dk) < 1e-14 * k:
            break
    return k


def _cf(x, Xi, dl):
    """cfv/cfh profile (2d/functions.c:787-799)."""
    h = (x - Xi >= 0).astype(float)
    return h * np.maximum(_sign(x - (Xi + dl)), (1 - np.cos((x - Xi) * math.pi / dl)) / 2)


def chiadj_vertical(x, ny, x_line, nadj, lam):
    """ChiAdj of a vertical influx line spanning every row (2d/functions.c:905-921):
    1 - cf(x, X - Nadj lam, Nadj lam) + cf(x, X, Nadj lam) on each row."""
    if nadj == 0:
        return np.ones((ny, x.size))
    dl = nadj * lam
    row = 1 - _cf(x, x_line - dl, dl) + _cf(x, x_line, dl)
    return np.tile(row, (ny, 1))


def area_kernels_vertical(x, y, kx, depth, x_line, Lbottom, Ltop):
    """newGam and SkewGam of a vertical line spanning every row (fun_area_generation,
    2d/functions.c:2991-3085): the group-velocity kernel of the x wavenumbers
    (make_1d_sym + real inverse transform), shifted to the line, its x derivative, a
    heaviside in y that leaves out the bottom/top damping zones, scaled by
    (2 pi)^2 / (dx dy).  Returned in [row y][column x] layout."""
    nx, ny = x.size, y.size
    dx, dy = x[1] - x[0], y[1] - y[0]
    ug_hat = exact_ug(kx, depth).astype(float)
    for idd, j in enumerate(range(nx - 1, nx // 2, -1), start=1):   # make_1d_sym
        ug_hat[j] = ug_hat[idd]
    ugx = np.fft.ifft(ug_hat).real
    ugx = np.roll(ugx, int(round((x_line - x[0]) / dx)))
    dug = np.fft.fft(ugx)
    d_hat = 1j * kx * dug
    for idd, j in enumerate(range(nx - 1, nx // 2, -1), start=1):   # make_1dcom_sym
        d_hat[j] = np.conj(d_hat[idd])
    dxg = np.fft.ifft(d_hat).real
    hb = np.ones(ny) if Lbottom == 0 else (y - (y[0] + Lbottom) >= 0).astype(float)
    ht = np.zeros(ny) if Ltop == 0 else (y - (y[ny - 1] - Ltop) >= 0).astype(float)
    heav = hb * (1 - ht)
    fact = (2 * math.pi) ** 2 / (dx * dy)
    return fact * heav[:, None] * ugx[None, :], fact * heav[:, None] * dxg[None, :]


def directional_signals(y, t, Hs, Tp, gamma, s_spread, depth, n_freq, n_dir, seed, ramp=2.0, mdir=0.0):
    """Seeded directional JONSWAP line signals on the influx line: n_freq x n_dir
    components, frequencies on the time grid's Fourier lines and cross-line
    wavenumbers k(omega) sin(theta) on the y grid's, cos^2s spreading about mdir,
    uniform random phases.  Returns (signal, skew signal) [ny][nt]: the elevation
    along the line and its quadrature, both with a cosine ramp of `ramp` s."""
    rng = np.random.default_rng(seed)
    ny, nt = y.size, t.size
    dt = t[1] - t[0]
    Ly = ny * (y[1] - y[0])
    wp = 2 * math.pi / Tp
    w = np.linspace(0.5 * wp, 3.0 * wp, n_freq)
    sig = np.where(w <= wp, 0.07, 0.09)
    S = (GRAV ** 2 / w ** 5) * np.exp(-1.25 * (wp / w) ** 4) * gamma ** np.exp(-((w - wp) ** 2) / (2 * sig ** 2 * wp ** 2))
    dw = w[1] - w[0]
    m0 = np.sum(S) * dw
    S *= (Hs / 4.0) ** 2 / m0
    th = np.linspace(-math.pi / 2, math.pi / 2, n_dir)
    D = np.cos((th - mdir) / 2) ** (2 * s_spread)
    dth = th[1] - th[0]
    D /= np.sum(D) * dth
    spec = np.zeros((ny, nt), dtype=complex)
    for m in range(n_freq):
        k = invers_omega(w[m], depth)
        n_w = int(round(w[m] * nt * dt / (2 * math.pi)))
        for d in range(n_dir):
            a = math.sqrt(2 * S[m] * D[d] * dw * dth)
            n_k = int(round(k * math.sin(th[d]) * Ly / (2 * math.pi))) % ny
            spec[n_k, (-n_w) % nt] += a * np.exp(1j * rng.uniform(0, 2 * math.pi))
    z = np.fft.ifft2(spec) * (ny * nt)   # sum_a a exp(i (ky y - w t + phi))
    r = np.clip(t / ramp, 0, 1) if ramp > 0 else np.ones(nt)
    r = 0.5 * (1 - np.cos(math.pi * r))
    return z.real * r[None, :], z.imag * r[None, :]


def reference_directional_components(t, Hs, Tp, gamma, s_spread, depth, seed):
    """The spectral components of the 2D set-up's jonswap_influx (2d/functions.c:2226-2446)
    for the time grid t: the first Nt/2 frequencies of freqspace over the time span, the
    wavenumber of each at `depth` (exact dispersion), amplitudes sqrt(2 S dw) of
    fun_jonswap's spectrum (normalised to Hs by the trapezoid m0), one direction each
    drawn from the cos^2s distribution (s_spread; None or inf: long-crested) by
    interpolating the inverse of its cumulative sum (natural cubic spline, as
    gsl_spline_eval), and uniform phases.  The reference draws the uniforms from
    srand(time(0)); here they come from the seeded splitmix64 stream (directions from
    seed 2 seed + 1, phases from 2 seed + 2).  Returns (a, w, k, theta, phi)."""
    from scipy.interpolate import CubicSpline
    from .decks import splitmix64_uniform
    nt = t.size
    nh = nt // 2
    ww = freqspace(float(t[-1] - t[0]), nt)[:nh]
    wp = 2 * math.pi / Tp
    fp = wp / (2 * math.pi)
    JS = np.zeros(nh)
    f = ww[1:] / (2 * math.pi)
    sig = np.where(ww[1:] <= wp, 0.07, 0.09)
    gp = np.exp(-0.5 * ((f / fp - 1) / sig) ** 2)
    JS[1:] = 0.0081 * GRAV ** 2 * (2 * math.pi) ** -4 * f ** -5 * np.exp(-(5.0 / 4.0) * (f / fp) ** -4) * gamma ** gp
    m0 = (np.sum(JS) - JS[0] / 2 - JS[-1] / 2) * (ww[1] - ww[0])
    a = np.sqrt(2 * (Hs ** 2 / 16) * JS / m0 * (ww[1] - ww[0]))
    th = -math.pi / 2 + np.arange(nh) * (math.pi / (nh - 1))
    if s_spread is None or not np.isfinite(s_spread):
        theta = np.zeros(nh)
    else:
        s = float(s_spread)
        coef = math.gamma(s + 1.0) / (math.sqrt(math.pi) * math.gamma(s + 0.5))
        cdf = np.cumsum(coef * np.cos(th) ** (2 * s))
        cdf = cdf / cdf[-1] + math.exp(-12.0) / math.pi * th
        theta = CubicSpline(cdf, th, bc_type="natural")(splitmix64_uniform(2 * seed + 1, nh))
    phi = 2 * math.pi * splitmix64_uniform(2 * seed + 2, nh)
    return a, ww, kappa_of_omega(ww, depth), theta, phi


def two_depth_operator(depth, kx, ky, omega_p, U=0.0, mdir=0.0):
    """Tables of the two-reference-depth operator (funOprt_DispInterpolation_2p,
    2d/functions.c:1534-1626): on 101 depths between the shallowest and deepest
    point, the weights (gam_min, gam_plus) that make the blend of the two reference
    phase speeds and squared frequencies exact at the local wavenumber of the peak
    frequency; a natural cubic spline in depth gives them per point.  The spectral
    tables are C^2 and Om^2 of the two reference depths."""
    from scipy.interpolate import CubicSpline
    d_min, d_max = float(depth.min()), float(depth.max())
    N = 101
    dD = (d_max - d_min) / (N - 1)
    DD = d_min + dD * np.arange(N)
    DD[-1] += 0.1 * dD

    def cp1(k, D):
        return math.sqrt(GRAV * D) + U if k == 0 else (math.copysign(1.0, k) * math.sqrt(GRAV * k * math.tanh(k * D)) + k * U) / k

    def om2(k, D):
        return (math.copysign(1.0, k) * math.sqrt(GRAV * k * math.tanh(k * D)) + k * U) ** 2

    gmin, gplus = np.empty(N), np.empty(N)
    for i in range(N):
        kap = invers_omega(omega_p, DD[i])
        cD, cm, cp = cp1(kap, DD[i]), cp1(kap, d_min), cp1(kap, d_max)
        oD, om_, op_ = om2(kap, DD[i]), om2(kap, d_min), om2(kap, d_max)
        det = cm * op_ - cp * om_
        gmin[i] = (op_ * cD - cp * oD) / det
        gplus[i] = (-om_ * cD + cm * oD) / det
    sm_, sp_ = CubicSpline(DD, gmin, bc_type="natural"), CubicSpline(DD, gplus, bc_type="natural")
    KX, KY = np.meshgrid(kx, ky)
    out = {"gam_min": sm_(depth), "gam_plus": sp_(depth)}
    for name, D in (("min", d_min), ("plus", d_max)):
        out[f"om2_{name}"] = exact_disp(KX, KY, D, mdir, 0.0, 0.0) ** 2
        out[f"csq_{name}"] = exact_cp(KX, KY, D) ** 2
    return out


def three_depth_operator(depth, kx, ky, omega_p, d_mid=None, U=0.0, mdir=0.0):
    """Tables of the three-reference-depth operator (funOprt_DispInterpolation_3p,
    2d/functions.c:1627-1762): on 100 depths between the shallowest and deepest point,
    the weights (gam_min, gam_mid, gam_plus) that make the blend of the three reference
    long-wave speeds, squared frequencies and phase speeds exact at the local
    wavenumber of the peak frequency (Cramer's rule with the reference's cofactors
    A..I); a natural cubic spline in depth gives them per point.  d_mid defaults to
    the mean of the extreme depths ("default" in the deck).  As for two depths, the
    peak wavenumber is the exact inverse of the dispersion relation."""
    from scipy.interpolate import CubicSpline
    d_min, d_max = float(depth.min()), float(depth.max())
    d_mid = (d_max + d_min) / 2 if d_mid is None else float(d_mid)
    N = 100
    dD = (d_max - d_min) / (N - 1)
    DD = d_min + dD * np.arange(N)
    DD[-1] += 0.1 * dD

    def cp1(k, D):
        return math.sqrt(GRAV * D) + U if k == 0 else (math.copysign(1.0, k) * math.sqrt(GRAV * k * math.tanh(k * D)) + k * U) / k

    def om2(k, D):
        return (math.copysign(1.0, k) * math.sqrt(GRAV * k * math.tanh(k * D)) + k * U) ** 2

    g = np.empty((3, N))
    c0m, c0c, c0p = math.sqrt(GRAV * d_min), math.sqrt(GRAV * d_mid), math.sqrt(GRAV * d_max)
    for i in range(N):
        kap = invers_omega(omega_p, DD[i])
        cD, cm, cc, cp = cp1(kap, DD[i]), cp1(kap, d_min), cp1(kap, d_mid), cp1(kap, d_max)
        oD, om_, oc, op_ = om2(kap, DD[i]), om2(kap, d_min), om2(kap, d_mid), om2(kap, d_max)
        c0D = math.sqrt(GRAV * DD[i])
        A = (oc * cp) - (op_ * cc)
        B = -(om_ * cp) + (op_ * cm)
        C = (om_ * cc) - (oc * cm)
        D = -(c0c * cp) + (c0p * cc)
        E = (c0m * cp) - (c0p * cm)
        F = -(c0m * cc) + (c0c * cm)
        G = (c0c * op_) - (c0p * oc)
        H = -(c0m * op_) + (c0p * om_)
        I = (c0m * oc) - (c0c * om_)
        det = c0m * A + c0c * B + c0p * C
        g[0, i] = (A * c0D + D * oD + G * cD) / det
        g[1, i] = (B * c0D + E * oD + H * cD) / det
        g[2, i] = (C * c0D + F * oD + I * cD) / det
    KX, KY = np.meshgrid(kx, ky)
    out = {}
    for r, name, D in ((0, "min", d_min), (1, "mid", d_mid), (2, "plus", d_max)):
        out[f"gam_{name}"] = CubicSpline(DD, g[r], bc_type="natural")(depth)
        out[f"om2_{name}"] = exact_disp(KX, KY, D, mdir, 0.0, 0.0) ** 2
        out[f"csq_{name}"] = exact_cp(KX, KY, D) ** 2
    out["_knots"] = (DD, g, (d_min, d_mid, d_max))
    return out


def kappa_of_omega(omega, depth):
    """Wavenumber of frequency omega at each depth (Newton on omega^2 = g k tanh(k d),
    vectorised, to rounding)."""
    d = np.asarray(depth, dtype=np.float64)
    k = omega / np.sqrt(GRAV * d)
    for _ in range(60):
        t = np.tanh(k * d)
        k = k - (GRAV * k * t - omega ** 2) / (GRAV * t + GRAV * k * d * (1 - t * t))
    return k


def log_reference_depths(depth, K):
    """K log-spaced reference depths over [min h, max h]."""
    dmin, dmax = float(np.min(depth)), float(np.max(depth))
    D = dmin * (dmax / dmin) ** (np.arange(K) / (K - 1))
    D[0], D[-1] = dmin, dmax
    return D


def k_reference_weights(depth, omega_p, D):
    """Per-point weights [K][...] of the K-reference operator (no counterpart in the
    reference): each point on its bracketing pair [D_j, D_j+1] with the two-depth
    weights of funOprt_DispInterpolation_2p (2d/functions.c:1534-1626) -- the blend of
    the pair's phase speeds and squared frequencies exact at the point's own depth
    for the wavenumber of the peak frequency there -- evaluated at the point itself
    instead of through a spline over 101 depth samples.  Weights of the other depths
    are zero."""
    h = np.asarray(depth, dtype=np.float64)
    K = len(D)
    j = np.clip(np.searchsorted(D, h, side="right") - 1, 0, K - 2)
    kap = kappa_of_omega(omega_p, h)

    def cp1(k, d):
        return np.sqrt(GRAV * np.tanh(k * d) / k)

    def om2(k, d):
        return GRAV * k * np.tanh(k * d)

    Da, Db = np.asarray(D)[j], np.asarray(D)[j + 1]
    cD, cm, cp = cp1(kap, h), cp1(kap, Da), cp1(kap, Db)
    oD, om_, op_ = om2(kap, h), om2(kap, Da), om2(kap, Db)
    det = cm * op_ - cp * om_
    w = np.zeros((K,) + h.shape)
    ia = np.indices(h.shape)
    w[(j,) + tuple(ia)] = (op_ * cD - cp * oD) / det
    w[(j + 1,) + tuple(ia)] = (-om_ * cD + cm * oD) / det
    return w


def with_k_operator(tb, D, gam):
    """A copy of a varying-bottom tables dict whose operator is the K-reference one:
    reference depths D (K), per-point weights gam [K][ny][nx]; the spectral tables are
    C^2 and Omega^2 of each depth, as for the two-depth operator.  The min/plus/mid
    tables are dropped (hw2d_tables takes one form or the other)."""
    out = {k: v for k, v in tb.items() if not (k.startswith(("gam_", "csq_", "om2_")))}
    KX, KY = np.meshgrid(tb["kx"], tb["ky"])
    K = len(D)
    out["nrefk"] = K
    out["gam_k"] = np.ascontiguousarray(np.asarray(gam, dtype=np.float64).reshape(K, -1))
    out["csq_k"] = np.ascontiguousarray(np.stack([(exact_cp(KX, KY, d) ** 2).ravel() for d in D]))
    out["om2_k"] = np.ascontiguousarray(np.stack([(exact_disp(KX, KY, d) ** 2).ravel() for d in D]))
    out["ref_depths"] = np.asarray(D, dtype=np.float64)
    return out


def plain_k_operator(tb, K=16):
    """The plain K-reference operator of a varying-bottom tables dict (log-spaced
    depths over the bottom's range, weights from k_reference_weights)."""
    depth = tb["depth"]
    D = log_reference_depths(depth, K)
    return with_k_operator(tb, D, k_reference_weights(depth, tb["wp"], D))


def shoal_bathymetry(x, y, deep=5.0, shallow=0.5, x1=100.0, x2=285.0, seed=0):
    """Depth 0.5-5 m: deep up to x1, a linear slope to `shallow` at x2, and a seeded
    Gaussian shoal on the slope; clipped to [shallow, deep]."""
    rng = np.random.default_rng(seed + 7919)
    X, Y = np.meshgrid(x, y)
    d = deep + (shallow - deep) * np.clip((X - x1) / (x2 - x1), 0.0, 1.0)
    xc = x1 + (x2 - x1) * rng.uniform(0.3, 0.6)
    yc = y[0] + (y[-1] - y[0]) * rng.uniform(0.3, 0.7)
    sig = 0.08 * (x[-1] - x[0])
    d -= 1.5 * np.exp(-((X - xc) ** 2 + (Y - yc) ** 2) / (2 * sig ** 2))
    return np.clip(d, shallow, deep)


def tables(nx=1024, ny=1024, Lx=300.0, Ly=300.0, depth=3.0, Hs=0.5, Tp=6.0, gamma=3.3, s_spread=10,
           n_freq=256, n_dir=64, t_end=300.0, dt=0.1, damp=30.0, x_line=45.0, nadj=1.0, model=2,
           propagation=0, seed=0, bathymetry="flat", shallow=0.5, walls=(), refl=0.5, breaking=False,
           kbc=0.8, tc=0.2, tchar=0.5, ninterp=2, influx_model="lines", device=0) -> dict:
    """All tables of a 2D deck (vertical influx line at x_line).  bathymetry "flat":
    depth everywhere (rhs_AB2_2DF_uv); "shoal": `depth` offshore sloping to
    `shallow` with a seeded shoal, two reference depths (rhs_AB2_2DB_uv), or three
    with ninterp=3 (HSSgen_3depth).
    breaking=True adds the kinematic-breaking tables of parambreak
    (2d/breaking.c:1-44) with the deck's KBC, TC, Tchar.
    influx_model "lines": n_freq x n_dir seeded components on the grids' Fourier lines
    (directional_signals); "reference": jonswap_influx's own model, Nt/2 components with
    one direction each (reference_directional_components), summed on the CUDA device
    `device`."""
    x = np.linspace(0.0, Lx, nx)          # fun_intervaltovector (2d/functions1.c:204)
    y = np.linspace(0.0, Ly, ny)
    kx = freqspace(x[-1] - x[0], nx)
    ky = freqspace(y[-1] - y[0], ny)
    KX, KY = np.meshgrid(kx, ky)
    c2d = exact_cp(KX, KY, depth)
    om = exact_disp(KX, KY, depth)
    l2d = om * om / GRAV
    cutfrac = {1: 2, 2: 4, 3: 6}[model]   # evolinfo.cutfrac (2d/functions.c:209-219)
    aal = aal2d(kx, ky, cutfrac)
    wall = None
    if walls:
        wall, cfw = wallchar2d(x, y, list(walls), refl, model)
        charac = fbdy2d(x, y, damp, damp, damp, damp, cfsa_wall=cfw, model=model)
    else:
        charac = fbdy2d(x, y, damp, damp, damp, damp)
    wp = 2 * math.pi / Tp
    var = None
    depth_field = None
    if bathymetry != "flat":
        depth_field = shoal_bathymetry(x, y, deep=depth, shallow=shallow,
                                       x1=x[0] + 0.33 * (x[-1] - x[0]), x2=x[0] + 0.95 * (x[-1] - x[0]), seed=seed)
        var = (two_depth_operator if ninterp == 2 else three_depth_operator)(depth_field, kx, ky, wp)
        var.pop("_knots", None)
    kp = invers_omega(wp, depth)
    cpeak = wp / kp                        # fun_exact_Cp1d_val(kp, depth at the influx line, 0)
    chi = chiadj_vertical(x, ny, x_line, nadj, 2 * math.pi / kp)
    newgam, skewgam = area_kernels_vertical(x, y, kx, depth, x_line, damp, damp)
    nt = int(round(t_end / dt)) + 1
    tsig = np.arange(nt) * dt
    if influx_model == "reference":
        # jonswap_influx's own model: Nt/2 components, one random direction each,
        # summed for every sample and line point on the device
        from .engine2d import directional_signal
        comps = reference_directional_components(tsig, Hs, Tp, gamma, s_spread, depth, seed)
        r = np.clip(tsig / 2.0, 0, 1)
        sig, sigs = directional_signal(0.0, dt, nt, y, y[0], comps, ramp_t=0.5 * (1 - np.cos(math.pi * r)),
                                       device=device)
    else:
        sig, sigs = directional_signals(y, tsig, Hs, Tp, gamma, s_spread, depth, n_freq, n_dir, seed)
    # The area kernel carries (2 pi)^2 / (dx dy) and integrates to that times dx along
    # x; scaling the elevation by dy / (2 pi)^2 makes the line generate the target
    # elevation (the reference reaches the same end by dividing the influx spectrum by
    # the transform of the area function, 2d/functions.c:3196-3214).
    scale = (y[1] - y[0]) / (2 * math.pi) ** 2
    sig, sigs = sig * scale, sigs * scale
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    extra = {k: f64(v) for k, v in var.items()} if var else {}
    if depth_field is not None:
        extra["depth"] = f64(depth_field)
    if breaking:
        if depth_field is None:
            depth_field_b = np.full((ny, nx), float(depth))
        else:
            depth_field_b = depth_field
        # pb.Char: cfSA (min with the wall's cfSAwall, 2d/functions.c:1960-1967), zero
        # where cfSA < 1 or ChiAdj < 1 (2d/breaking.c:10-21)
        cf = cfsa2d(x, y, damp, damp, damp, damp)
        if wall is not None:
            cf = np.minimum(cf, cfw)
        brchar = np.where((cf < 1) | (chi < 1), 0.0, cf)
        extra.update(breaking=1, bathy=f64(-depth_field_b), brchar=f64(brchar), dx=float(x[1] - x[0]),
                     dy=float(y[1] - y[0]), max_eta_init=Hs / 2.0 * 0.9, tstar=tchar * Tp,
                     rsearch=2 * math.pi / kp / 4.0, kbc=float(kbc), tc=float(tc), delb=1.5, cur_u=0.0,
                     t0=0.0)
    if wall is not None:
        extra["wallchar"] = f64(wall)
        extra["refl_coef"] = float(refl)
    extra.setdefault("dx", float(x[1] - x[0]))
    extra.setdefault("dy", float(y[1] - y[0]))
    # what the output stage writes to Constant_01.dat besides the grids (print_xt)
    extra.setdefault("bathy", f64(-(depth_field if depth_field is not None else np.full((ny, nx), float(depth)))))
    cf_out = cfsa2d(x, y, damp, damp, damp, damp)
    if wall is not None:
        cf_out = np.minimum(cf_out, cfw)
    extra.update(cfsa=f64(cf_out), hs=float(Hs), kp=float(kp), wp=float(wp))
    return dict(**extra, nx=nx, ny=ny, model=model, propagation=propagation, cpeak=float(cpeak), kx=f64(kx), ky=f64(ky),
                c2d=f64(c2d), l2d=f64(l2d), aal=f64(aal), charac=f64(charac), chiadj=f64(chi),
                newgam=f64(newgam), skewgam=f64(skewgam), nt=nt, tsig=f64(tsig), sig=f64(sig), sigskew=f64(sigs),
                dt_out=dt, x=x, y=y)


def outputs(tb, tout, npartition=1, gauges=None, uv_every_sample=False, chiadjphi=None) -> dict:
    """The output-stage arguments of ode_solver_uv for a tables dict (keyword
    arguments of Engine2D.run_outputs): output times, partitions, the grids and the
    Constant_01.dat tables, gauges as (x, y) pairs."""
    tout = np.asarray(tout, dtype=np.float64)
    return dict(tout=tout, dt=float(tout[1] - tout[0]) if tout.size > 1 else 0.0, npartition=int(npartition),
                x=tb["x"], y=tb["y"], dx=tb["dx"], dy=tb["dy"], kx=tb["kx"], ky=tb["ky"], bathy=tb["bathy"],
                cfsa=tb["cfsa"], chiadjphi=chiadjphi, hs=tb["hs"], kp=tb["kp"], wp=tb["wp"], gauges=gauges,
                uv_every_sample=uv_every_sample)


def config5(seed=0, bathymetry="shoal", **kw) -> dict:
    """The 2D workload: 1024 x 1024 on 300 m x 300 m, depth 5 m offshore sloping to
    0.5 m with a seeded shoal (two reference depths; bathymetry="flat" gives a flat
    3 m bottom and no wall), a harbour breakwater (x 200-206 m, y 90-210 m) of
    reflection coefficient 0.5, directional JONSWAP Hs 0.5 m Tp 6 s gamma 3.3,
    cos^2s spreading s = 10, 256 x 64 seeded components, HS2 with kinematic
    breaking (KBC 0.8, TC 0.2, Tchar 0.5), 30 m damping
    zones, influx line at x = 45 m."""
    if bathymetry == "flat":
        return tables(seed=seed, **kw)
    kw.setdefault("breaking", True)
    kw.setdefault("depth", 5.0)
    kw.setdefault("walls", ((200.0, 90.0, 206.0, 210.0),))
    kw.setdefault("refl", 0.5)
    return tables(seed=seed, bathymetry=bathymetry, **kw)
