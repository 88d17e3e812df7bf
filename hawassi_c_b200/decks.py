"""Seeded synthetic decks in the reference's input format.

A deck is a directory holding ``input.txt`` (the fixed-layout key/value file read
positionally by 1d/read_input.c:1-60 and 1d/influx_lib.c:1-109), and, as needed,
``influx.dat`` (two columns t, eta: ``wavename = user_defined``), ``bath.dat``
(one depth per grid point) and ``gauges.dat``.  Both the device engine and the
CPU oracle read the same files, so seeded realisations are reproducible on both
sides (the reference draws its own JONSWAP phases from srand(time(0))).

Phases come from a counter-based splitmix64 stream: component j of seed s uses
the j-th output of the stream started at s, independent of the platform.
"""
import math
import os

import numpy as np

G = 9.80665

_INPUT = """&INFLUX_SIGNAL
wavename = {wavename}
initial  = {initial}

&IF wavename jonswap
T0\t\t= {T0}
Tend\t \t= {Tend}
dt \t\t= {dt}
Tp \t\t= {Tp}
Hs\t\t= {Hs}
gamma \t \t= {gamma}

&SPATIAL
Xstart\t\t= {Xstart}
Xend\t\t= {Xend}
Xinflux\t\t= {Xinflux}
dx\t\t= {dx}
Damp \t\t= {dampL} {dampR}
bathymetry\t= {bath}
depth \t\t= {depth}
adjcoef\t\t= {adjcoef}

&EVOL_MODEL
dynamics\t= {model}
breaking\t= {breaking}
friction \t= no
influxing \t= {influxing}
propagation \t= {propagation}
kinematic \t= {kinematic}
ngauge \t\t= {ngauge}
npartition \t= {npartition}

&IF BREAKING
initiation \t= {kbc}
termination = {tc} {tchar}

&IF KINEMATIC
xstart\t\t= {kx1}
xend\t\t= {kx2}
nsurf \t\t= {nsurf}
ndeep \t\t= {ndeep}

&MORE OPTIONS FOR EXPERT ONLY
cutfrac\t\t  = {cutfrac}
mid_depth_ref = default
min_zsurf\t  = default
max_zsurf \t  = default
ramp_influx \t= {ramp}
wall \t\t= no
walltype \t= 1 30 1

&INPUT COUPLING MODULE
coupling \t= no ../foc/output
overlay \t= 30 40
"""


def splitmix64_uniform(seed, count):
    """count uniforms in [0, 1) from the splitmix64 stream started at seed."""
    out = np.empty(count)
    s = seed & 0xFFFFFFFFFFFFFFFF
    mask = 0xFFFFFFFFFFFFFFFF
    for i in range(count):
        s = (s + 0x9E3779B97F4A7C15) & mask
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z = z ^ (z >> 31)
        out[i] = (z >> 11) * (1.0 / 9007199254740992.0)
    return out


def jonswap_density(omega, Hs, Tp, gamma):
    """JONSWAP spectral density S(omega) (m^2 s), alpha rescaled to the requested Hs."""
    wp = 2 * math.pi / Tp
    sigma = np.where(omega <= wp, 0.07, 0.09)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        pm = G ** 2 / omega ** 5 * np.exp(-1.25 * (wp / omega) ** 4)
        r = np.exp(-((omega - wp) ** 2) / (2 * sigma ** 2 * wp ** 2))
        S = pm * gamma ** r
    S = np.nan_to_num(S)
    dw = omega[1] - omega[0]
    m0 = S.sum() * dw
    return S * (Hs ** 2 / 16.0) / m0 if m0 > 0 else S


def jonswap_signal(T_end, n_samples, n_lines, Hs, Tp, gamma, seed):
    """eta(t) at n_samples equispaced times on [0, T_end]: a sum of n_lines harmonic
    components on the frequency grid j*2*pi/T_end with JONSWAP amplitudes and
    seeded uniform phases, rescaled so that 4*std(eta) = Hs."""
    t = np.linspace(0.0, T_end, n_samples)
    dw = 2 * math.pi / T_end
    omega = dw * np.arange(1, n_lines + 1)
    amp = np.sqrt(2 * jonswap_density(omega, Hs, Tp, gamma) * dw)
    phase = 2 * math.pi * splitmix64_uniform(seed, n_lines)
    eta = np.zeros_like(t)
    for j in range(0, n_lines, 256):
        sl = slice(j, j + 256)
        eta += (amp[sl, None] * np.cos(omega[sl, None] * t[None, :] + phase[sl, None])).sum(axis=0)
    std = eta.std()
    if std > 0:
        eta *= Hs / (4 * std)
    return t, eta


def dx_for(length, nx):
    """dx such that the reference's int(length/dx)+1 gives exactly nx (even)."""
    return length / (nx - 0.5)


def write_deck(path, nx, length=None, xstart=0.0, xinflux=None, depth=1.0, bath=None, model="HS2",
               breaking=False, T_end=100.0, n_samples=2048, n_lines=1024, Hs=0.10, Tp=2.0, gamma=3.3,
               seed=0, damp=(10.0, 10.0), adjcoef=0.5, propagation="Uni+", influxing="Area",
               kbc=0.8, tc=0.2, tchar=0.5, cutfrac="default", ramp="yes 4", wavename="user_defined",
               initial="zero", initial_wave=None, gauges=(), dt=0.02, npartition=1, kinematic=False,
               kin_window=(40.0, 60.0), nsurf=50, ndeep=40):
    """Write one deck directory.  bath: None for flat depth, or an array of nx depths.
    kinematic: the kinematics output on the overlay window kin_window (x range, m)
    with nsurf surface and ndeep deep levels (read_kinematics, 1d/functions.c:3555)."""
    os.makedirs(path, exist_ok=True)
    length = float(length if length is not None else 0.05 * nx)
    xend = xstart + length
    if xinflux is None:
        xinflux = xstart + 0.1 * length
    fields = dict(
        wavename=wavename, initial=initial, T0=0, Tend=repr(float(T_end)), dt=repr(float(dt)), Tp=repr(float(Tp)),
        Hs=repr(float(Hs)), gamma=repr(float(gamma)), Xstart=repr(float(xstart)), Xend=repr(float(xend)),
        Xinflux=repr(float(xinflux)), dx=repr(dx_for(length, nx)), dampL=repr(float(damp[0])),
        dampR=repr(float(damp[1])), bath="flat" if bath is None else "user_defined", depth=repr(float(depth)),
        adjcoef=repr(float(adjcoef)), model=model, breaking="yes" if breaking else "no", influxing=influxing,
        propagation=propagation, ngauge=len(gauges), npartition=int(npartition), kbc=repr(float(kbc)), tc=repr(float(tc)),
        tchar=repr(float(tchar)), cutfrac=cutfrac, ramp=ramp, kinematic="yes" if kinematic else "no",
        kx1=repr(float(kin_window[0])), kx2=repr(float(kin_window[1])), nsurf=int(nsurf), ndeep=int(ndeep))
    with open(os.path.join(path, "input.txt"), "w") as f:
        f.write(_INPUT.format(**fields))
    if wavename == "user_defined":
        t, eta = jonswap_signal(T_end, n_samples, n_lines, Hs, Tp, gamma, seed)
        with open(os.path.join(path, "influx.dat"), "w") as f:
            for a, b in zip(t, eta):
                f.write(f"{float(a)!r} {float(b)!r}\n")
    if bath is not None:
        bath = np.asarray(bath, dtype=np.float64)
        assert bath.size == nx
        with open(os.path.join(path, "bath.dat"), "w") as f:
            for v in bath:
                f.write(f"{float(v)!r}\n")
    if initial == "user_defined":
        w = np.asarray(initial_wave, dtype=np.float64)
        with open(os.path.join(path, "initial.dat"), "w") as f:
            for a, b in w:
                f.write(f"{float(a)!r} {float(b)!r}\n")
    with open(os.path.join(path, "gauges.dat"), "w") as f:
        for gx in gauges:
            f.write(f"{float(gx)!r}\n")
    return path


def slope_bathymetry(nx, length, xstart=0.0, h0=1.0, x_toe=150.0, slope=1.0 / 30.0, h_min=0.05):
    """Flat depth h0 up to x_toe, then a linear slope down to h_min (a shelf after)."""
    x = xstart + np.arange(nx) * (length / (nx - 1))
    return np.maximum(h0 - np.maximum(x - x_toe, 0.0) * slope, h_min)


def bump_bathymetry(nx, length, seed, n_bumps=8, h_min=0.05, h_max=2.0):
    """Depth in [h_min, h_max]: a base depth plus n_bumps seeded Gaussian bumps/troughs."""
    u = splitmix64_uniform(seed * 7919 + 17, 4 * n_bumps + 1)
    x = np.arange(nx) * (length / (nx - 1))
    h = np.full(nx, h_min + (h_max - h_min) * (0.4 + 0.4 * u[0]))
    for b in range(n_bumps):
        c = length * u[1 + 4 * b]
        w = length * (0.02 + 0.1 * u[2 + 4 * b])
        a = (h_max - h_min) * (u[3 + 4 * b] - 0.5) * 0.8
        h += a * np.exp(-((x - c) / w) ** 2)
    return np.clip(h, h_min, h_max)


def config1_deck(path, seed=0, T_end=100.0, nx=4096):
    """1D plain: L=200 m, Nx=4096, flat 1 m, HS2, no breaking, JONSWAP Hs 0.10 / Tp 2.0 /
    gamma 3.3 with 1024 lines (2048 influx samples), influx at x=20 m, 10 m damping zones."""
    return write_deck(path, nx=nx, length=200.0, xinflux=20.0, depth=1.0, model="HS2", breaking=False,
                      T_end=T_end, n_samples=2048, n_lines=1024, Hs=0.10, Tp=2.0, gamma=3.3, seed=seed,
                      damp=(10.0, 10.0), adjcoef=0.5)


def ensemble_member_params(seed):
    """The drawn parameters of ensemble member `seed`: Nx from {2048,4096,8192,16384},
    L=0.05*Nx, flat depth U[0.5,2], JONSWAP Hs U[0.05,0.20], Tp U[1.5,3.0], gamma U[1,5]."""
    u = splitmix64_uniform(1_000_003 * (seed + 1), 6)
    nx = [2048, 4096, 8192, 16384][min(int(u[0] * 4), 3)]
    return dict(nx=nx, length=0.05 * nx, depth=0.5 + 1.5 * u[1], Hs=0.05 + 0.15 * u[2], Tp=1.5 + 1.5 * u[3],
                gamma=1.0 + 4.0 * u[4])


def ensemble_member_deck(path, seed, T_end=100.0, breaking=True):
    """One member of the batched ensemble (parameters of ensemble_member_params), HS2."""
    pm = ensemble_member_params(seed)
    nx, depth, Hs, Tp, gamma, length = pm["nx"], pm["depth"], pm["Hs"], pm["Tp"], pm["gamma"], pm["length"]
    return write_deck(path, nx=nx, length=length, xinflux=0.1 * length, depth=depth, model="HS2",
                      breaking=breaking, T_end=T_end, n_samples=2048, n_lines=1024, Hs=Hs, Tp=Tp, gamma=gamma,
                      seed=seed, damp=(0.05 * length, 0.05 * length), adjcoef=0.5)


def config2_deck(path, seed=0, T_end=200.0, nx=16384, length=400.0):
    """1D varying bathymetry with breaking: L=400 m, Nx=16384, 1.0 m flat up to x=150 m,
    then a 1:30 slope to 0.05 m; HS3; breaking KBC 0.8, TC 0.2, Tchar 0.5; JONSWAP
    Hs 0.15 m, Tp 2.5 s, gamma 3.3 with seeded phases; influx at x=20 m."""
    bath = slope_bathymetry(nx, length, h0=1.0, x_toe=150.0, slope=1.0 / 30.0, h_min=0.05)
    return write_deck(path, nx=nx, length=length, xinflux=20.0, depth=1.0, bath=bath, model="HS3", breaking=True,
                      T_end=T_end, n_samples=2048, n_lines=1024, Hs=0.15, Tp=2.5, gamma=3.3, seed=seed,
                      damp=(10.0, 10.0), adjcoef=0.5, kbc=0.8, tc=0.2, tchar=0.5)


def config4_deck(path, seed=0, T_end=100.0, nx=16384, length=400.0):
    """Random bathymetry for the learned depth operator: L=400 m, Nx=16384, depth in
    [0.05, 2.0] m from 8 seeded Gaussian bumps/troughs, HS2, JONSWAP influx."""
    bath = bump_bathymetry(nx, length, seed, n_bumps=8, h_min=0.05, h_max=2.0)
    u = splitmix64_uniform(31 * seed + 5, 3)
    return write_deck(path, nx=nx, length=length, xinflux=20.0, depth=float(bath.max()), bath=bath, model="HS2",
                      breaking=False, T_end=T_end, n_samples=2048, n_lines=1024, Hs=0.05 + 0.1 * u[0],
                      Tp=1.5 + 1.5 * u[1], gamma=1.0 + 4.0 * u[2], seed=seed, damp=(10.0, 10.0), adjcoef=0.5)
