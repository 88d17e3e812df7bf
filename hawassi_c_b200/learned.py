"""Learned depth operator (no counterpart in the reference).

The plain varying-depth operator HSS interpolates the exact dispersion over 16
reference depths (each grid point on its bracketing pair).  The learned operator
keeps K = 4 reference depths and lets a small per-point network pick the blend
weights (softmax over the 4), so HSS needs ceil(4/2) + 4 = 6 transforms instead of
8 + 16 = 24.  The network sees 5 features per point -- the depth and the depth
smoothed at three scales (2, 8, 32 m), each as its position on the log scale of
the 4 reference depths, and the local dominant wavenumber as log(kappa_d h) -- and is trained so that the blended phase speed sum_j w_j C^2(kappa, D_j)
matches the 16-reference operator's at 8 wavenumbers spanning the point's
dominant band [0.6 kappa_d, 2 kappa_d].  The dominant band comes from fields the
plain 16-reference method produced (local wavenumber of eta by the Hilbert
transform, linear dispersion where no wave has arrived yet).

Training (forward, backward, Adam) and inference run on the GPU through the C ABI
(hw_mlp_*); the plain 16-reference run is the fallback (a periodic shadow step
measures the eta error of each member and switches it when above a threshold) and
the judge of the error.
"""
import ctypes
import math
import os

import numpy as np

from . import engine as _eng

G = 9.80665
BAND = np.array([0.6, 0.75, 0.9, 1.0, 1.1, 1.3, 1.6, 2.0])
K_LEARN = 4
K_PLAIN = 16
SCALES_M = (2.0, 8.0, 32.0)


def csq(kappa, depth):
    """C^2(kappa, d) = g tanh(kappa d) / kappa (exact dispersion, kappa > 0)."""
    kappa = np.asarray(kappa, dtype=np.float64)
    return G * np.tanh(kappa * depth) / kappa


def reference_depths(depth, K):
    """K log-spaced reference depths over [min h, max h] (the K-reference operator's)."""
    dmin, dmax = float(np.min(depth)), float(np.max(depth))
    D = dmin * (dmax / dmin) ** (np.arange(K) / (K - 1))
    D[0], D[-1] = dmin, dmax
    return D


def kappa_linear(omega, depth):
    """Wavenumber of frequency omega at depth d (Newton on omega^2 = g k tanh(k d))."""
    d = np.asarray(depth, dtype=np.float64)
    k = omega / np.sqrt(G * d)
    for _ in range(50):
        t = np.tanh(k * d)
        f = G * k * t - omega ** 2
        df = G * t + G * k * d * (1 - t * t)
        k = k - f / df
    return k


def smooth(a, dx, sigma):
    """Gaussian smoothing (periodic, by FFT) with standard deviation sigma (m)."""
    n = a.size
    kk = 2 * np.pi * np.fft.fftfreq(n, d=dx)
    return np.fft.ifft(np.fft.fft(a) * np.exp(-0.5 * (kk * sigma) ** 2)).real


def local_wavenumber(eta, dx, fallback, rel_amp=0.2):
    """Local wavenumber of eta from its Hilbert transform (smoothed); where the local
    amplitude is below rel_amp of the largest, the fallback field is used."""
    n = eta.size
    e = eta - eta.mean()
    H = np.fft.ifft(-1j * np.sign(np.fft.fftfreq(n)) * np.fft.fft(e)).real
    ge, gH = np.gradient(e, dx), np.gradient(H, dx)
    amp2 = e * e + H * H
    num = smooth(e * gH - H * ge, dx, 4.0)
    den = smooth(amp2, dx, 4.0)
    k = np.where(den > 0, num / np.maximum(den, 1e-300), 0.0)
    amp = np.sqrt(np.maximum(smooth(amp2, dx, 4.0), 0))
    ok = (amp > rel_amp * amp.max()) & (k > 0.2 * fallback) & (k < 5 * fallback)
    return np.where(ok, k, fallback)


def features(depth, dx, kdom):
    """(Nx, 5) float32 features.  The depth h and h smoothed at 2, 8 and 32 m enter as
    their position on the log scale of the 4 reference depths (0 at the shallowest
    reference, 3 at the deepest), the dominant band as log(kappa_dom * h): the blend
    weights are then one function of these for every bathymetry."""
    D = reference_depths(depth, K_LEARN)
    scale = np.log(D[-1] / D[0]) / (K_LEARN - 1) if D[-1] > D[0] else 1.0
    hs = [depth] + [np.maximum(smooth(depth, dx, s), 1e-3) for s in SCALES_M]
    f = [np.log(h / D[0]) / scale - 1.5 for h in hs] + [np.log(kdom * depth)]
    return np.stack(f, axis=1).astype(np.float32)


def records(depth, dx, kdom, D16, gam16, D4):
    """(Nx, 45) float32 training records: features, G[m][j] = C^2(kappa_m, D4_j),
    T[m] = sum_j gam16_j C^2(kappa_m, D16_j) (the 16-reference operator's)."""
    Nx = depth.size
    kap = kdom[:, None] * BAND[None, :]                        # (Nx, 8)
    Gm = np.stack([csq(kap, d) for d in D4], axis=2)            # (Nx, 8, 4)
    T = np.zeros((Nx, BAND.size))
    for j, d in enumerate(D16):
        T += gam16[j][:, None] * csq(kap, d)
    R = np.concatenate([features(depth, dx, kdom), Gm.reshape(Nx, -1), T], axis=1)
    return R.astype(np.float32)


class MLP:
    """The per-point network on the GPU (hw_mlp_*)."""

    def __init__(self, seed=0, device=0):
        L = _eng.load_library()
        self._h = L.hw_mlp_create(seed, device)
        if not self._h:
            raise _eng.EngineError(L.hw_mlp_last_error(None).decode())
        n = [ctypes.c_int() for _ in range(5)]
        self.rec = L.hw_mlp_sizes(*[ctypes.byref(v) for v in n])
        self.n_in, self.n_hidden, self.n_out, self.n_band, self.n_params = [v.value for v in n]

    def close(self):
        if self._h:
            _eng.load_library().hw_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise _eng.EngineError(f"{what}: " + _eng.load_library().hw_mlp_last_error(self._h).decode())

    @staticmethod
    def _fp(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))

    def params(self):
        p = np.zeros(self.n_params, dtype=np.float32)
        self._check(_eng.load_library().hw_mlp_get_params(self._h, self._fp(p)), "get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(_eng.load_library().hw_mlp_set_params(self._h, self._fp(p)), "set_params")

    def grad(self, recs):
        r = np.ascontiguousarray(recs, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        self._check(_eng.load_library().hw_mlp_grad(self._h, self._fp(r), r.shape[0], self._fp(g), self._fp(loss)),
                    "grad")
        return float(loss[0]), g

    def train(self, recs, epochs=20, batch=4096, lr=3e-3):
        r = np.ascontiguousarray(recs, dtype=np.float32)
        losses = np.zeros(epochs, dtype=np.float32)
        self._check(_eng.load_library().hw_mlp_train(self._h, self._fp(r), r.shape[0], epochs, batch, lr,
                                                      self._fp(losses)), "train")
        return losses

    def infer(self, feats):
        f = np.ascontiguousarray(feats, dtype=np.float32)
        w = np.zeros((self.n_out, f.shape[0]))
        self._check(_eng.load_library().hw_mlp_infer(self._h, self._fp(f), f.shape[0],
                                                      w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "infer")
        return w


def eta_of(y, nx):
    return np.fft.ifft(y[:nx] + 1j * y[nx:2 * nx]).real


def member_fields(deck, y, omega_p):
    """depth, dx, dominant wavenumber field of one member from a plain-run state y."""
    depth = _eng.deck_table(deck, "depth")
    dx = float(_eng.deck_table(deck, "dx")[0])
    kfall = kappa_linear(omega_p, depth)
    eta = eta_of(y, depth.size)
    if not np.all(np.isfinite(eta)):
        # the plain run diverged (waves steepening over the shallowest bumps with no
        # breaking): its fields carry no band information, use linear dispersion
        return depth, dx, kfall
    kdom = local_wavenumber(eta, dx, kfall)
    return depth, dx, kdom


def training_records(decks, t_run, stride=1, device=0):
    """Run the plain 16-reference method on the decks (one batched launch) for t_run
    seconds and build the training records from the fields it produced."""
    plain = _eng.Engine(decks, eps_abs=1e-8, eps_rel=1e-6, nref=K_PLAIN, device=device)
    plain.run_to_time(t_run)
    out = []
    for m, d in enumerate(decks):
        _, _, y = plain.state(m)
        omega_p = float(_eng.deck_table(d, "nu_peak")[0])
        depth, dx, kdom = member_fields(d, y, omega_p)
        gam16 = _eng.deck_table(d, "gamK", nref=K_PLAIN).reshape(K_PLAIN, -1)
        R = records(depth, dx, kdom, reference_depths(depth, K_PLAIN), gam16, reference_depths(depth, K_LEARN))
        out.append(R[::stride])
    plain.close()
    return np.concatenate(out, axis=0)


def learned_weights(mlp, deck, kdom=None):
    """Per-point weights [4][Nx] and the 4 reference depths for a deck."""
    depth = _eng.deck_table(deck, "depth")
    dx = float(_eng.deck_table(deck, "dx")[0])
    if kdom is None:
        kdom = kappa_linear(float(_eng.deck_table(deck, "nu_peak")[0]), depth)
    return mlp.infer(features(depth, dx, kdom)), reference_depths(depth, K_LEARN)


def install(eng, decks, weights):
    """Install per-member (weights, depths) into an engine created with nref = 4."""
    for m, (w, D) in enumerate(weights):
        eng.set_operator_weights(m, D, w)


class ShadowedEnsemble:
    """Learned-operator ensemble with the plain 16-reference method as fallback: every
    `period` output samples each active member is copied into the plain engine, both
    advance one sample, and a member whose eta differs by more than `threshold`
    (relative L2) continues on the plain operator from then on."""

    def __init__(self, decks, weights, period=20, threshold=1e-3, device=0, **kw):
        self.decks = list(decks)
        self.learned = _eng.Engine(self.decks, nref=K_LEARN, device=device, **kw)
        install(self.learned, self.decks, weights)
        self.plain = _eng.Engine(self.decks, nref=K_PLAIN, device=device, **kw)
        self.period, self.threshold = period, threshold
        self.fallback = np.zeros(len(self.decks), dtype=bool)
        self.i = 0
        self.checks = []

    def advance(self, n_samples):
        target = self.i + n_samples
        while self.i < target:
            nxt = min(target, (self.i // self.period + 1) * self.period)
            stops = [nxt if not f else -1 for f in self.fallback]
            self.learned.run_members(stops)
            fb = [nxt if f else -1 for f in self.fallback]
            if self.fallback.any():
                self.plain.run_members(fb)
            self.i = nxt
            if self.i % self.period == 0:
                self._shadow_check()

    def _shadow_check(self):
        active = [m for m in range(len(self.decks)) if not self.fallback[m]]
        for m in active:
            t, h, y = self.learned.state(m)
            self.plain.set_state(t, h, y, member=m, i_out=self.i)
        stops = [self.i + 1 if m in active else -1 for m in range(len(self.decks))]
        self.plain.run_members(stops)
        self.learned.run_members(stops)
        self.i += 1
        for m in active:
            nx = self.learned.nx[m]
            el = eta_of(self.learned.state(m)[2], nx)
            ep = eta_of(self.plain.state(m)[2], nx)
            err = float(np.linalg.norm(el - ep) / max(np.linalg.norm(ep), 1e-300))
            self.checks.append((self.i, m, err))
            if err > self.threshold:
                self.fallback[m] = True
                t, h, y = self.plain.state(m)
                self.plain.set_state(t, h, y, member=m, i_out=self.i)


def train_staged(mlp, recs, epochs=200, batch=4096, lr0=3e-3, stages=4):
    """Adam in `stages` equal rounds with the learning rate halved after each (a
    step-wise decay: the last rounds refine what the first ones found)."""
    out = []
    for k in range(stages):
        out.append(mlp.train(recs, epochs=max(1, epochs // stages), batch=batch, lr=lr0 * 0.5 ** k))
    return np.concatenate(out)


PARAMS_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "learned_k4.npy")


def load_mlp(path=PARAMS_FILE, device=0):
    """The network trained by pipeline(save=...), on the device (None when absent)."""
    if not os.path.exists(path):
        return None
    mlp = MLP(device=device)
    mlp.set_params(np.load(path).astype(np.float32))
    return mlp


def compare_on_ensemble(mlp, decks, t_warm=0.5, t_end=3.0, device=0):
    """Learned K = 4 ensemble against the plain 16-reference ensemble on the same
    decks: simulated seconds per wall second of each over [t_warm, t_end] (device
    time, CUDA events on the engines' own streams) and the eta relative L2 error of
    every learned member at t_end against its plain run."""
    import torch
    out = {}
    runs = {}
    for name, K in (("plain", K_PLAIN), ("learned", K_LEARN)):
        eng = _eng.Engine(decks, eps_abs=1e-8, eps_rel=1e-6, nref=K, device=device)
        if K == K_LEARN:
            install(eng, decks, [learned_weights(mlp, d) for d in decks])
        st = torch.cuda.Stream(device=device)
        eng.set_stream(st.cuda_stream)
        eng.run_to_time(t_warm)
        s0 = sum(eng.state(m)[0] for m in range(eng.members))
        r0 = sum(eng.stats(m)["rhs_calls"] for m in range(eng.members))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        eng.run_to_time(t_end, sync=False)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        s1 = sum(eng.state(m)[0] for m in range(eng.members))
        out[f"{name}_sim_s_per_wall_s"] = (s1 - s0) / (ms / 1e3)
        out[f"{name}_rhs_calls"] = sum(eng.stats(m)["rhs_calls"] for m in range(eng.members)) - r0
        runs[name] = [eta_of(eng.state(m)[2], eng.nx[m]) for m in range(eng.members)]
        eng.close()
    err = [float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)) for a, b in zip(runs["learned"], runs["plain"])]
    out.update(speedup=out["learned_sim_s_per_wall_s"] / out["plain_sim_s_per_wall_s"],
               eta_err_median=float(np.median(err)), eta_err_max=float(np.max(err)), members=len(decks),
               window_s=[t_warm, t_end])
    return out


# ---------------------------------------------------------------- the 2D variant
def smooth2d(a, dx, dy, sigma):
    """Isotropic Gaussian smoothing of a [ny][nx] field (periodic, by FFT), standard
    deviation sigma (m)."""
    ny, nx = a.shape
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=dx)
    ky = 2 * np.pi * np.fft.fftfreq(ny, d=dy)
    g = np.exp(-0.5 * sigma ** 2 * (ky[:, None] ** 2 + kx[None, :] ** 2))
    return np.fft.ifft2(np.fft.fft2(a) * g).real


def features2d(depth, dx, dy, kdom):
    """(ny*nx, 5) float32 features of a 2D bottom, the 1D features' definitions with the
    smoothing isotropic in the plane: h and h smoothed at 2, 8 and 32 m as positions
    on the log scale of the 4 reference depths, and log(kappa_dom h)."""
    D = reference_depths(depth, K_LEARN)
    scale = np.log(D[-1] / D[0]) / (K_LEARN - 1) if D[-1] > D[0] else 1.0
    hs = [depth] + [np.maximum(smooth2d(depth, dx, dy, s), 1e-3) for s in SCALES_M]
    f = [(np.log(h / D[0]) / scale - 1.5).ravel() for h in hs] + [np.log(kdom * depth).ravel()]
    return np.stack(f, axis=1).astype(np.float32)


def learned_tables2d(mlp, tb):
    """A 2D varying-bottom tables dict (decks2d.tables) with the learned K = 4 operator:
    the network's per-point softmax weights over 4 log-spaced reference depths, the
    dominant wavenumber from linear dispersion at the peak frequency.  The network is
    the 1D one: the blend it picks is a function of the local depth features and
    kappa_dom h, which the 2D bottom defines the same way."""
    from . import decks2d
    depth = tb["depth"]
    dx, dy = float(tb["dx"]), float(tb["dy"])
    kdom = kappa_linear(float(tb["wp"]), depth)
    w = mlp.infer(features2d(depth, dx, dy, kdom))
    return decks2d.with_k_operator(tb, reference_depths(depth, K_LEARN), w)


def wave_field_2d(tb, seed=0, hs_frac=0.25):
    """A sea state filling the whole 2D domain, as the initial state of a comparison:
    eta a seeded sum of random-phase waves of significant height hs_frac times the
    deck's (a quarter by default: no wave breaks over the shallowest bottom), their
    wavenumbers in [0.5 kp, 2 kp] and directions within 45 degrees of the x axis
    (kp of the peak period at the offshore depth), u = v = 0, in the spectral state
    layout [Re eta^ | Im eta^ | Re u^ | Im u^ | Re v^ | Im v^] (FFTW order) filtered by
    the anti-aliasing mask.  Unlike a start from rest, the waves cover the varying
    bottom from the first step, so a short window sees the depth operator everywhere."""
    rng = np.random.default_rng(seed)
    nx, ny = tb["nx"], tb["ny"]
    kx, ky = np.asarray(tb["kx"]), np.asarray(tb["ky"])
    kp = float(tb["kp"])
    KX, KY = np.meshgrid(kx, ky)
    kk = np.hypot(KX, KY)
    ang = np.abs(np.arctan2(KY, KX))
    band = (kk > 0.5 * kp) & (kk < 2.0 * kp) & (ang < np.pi / 4)
    spec = np.where(band, np.exp(-0.5 * ((kk - kp) / (0.3 * kp)) ** 2), 0.0)
    ehat = spec * np.exp(2j * np.pi * rng.random(spec.shape))
    eta = np.fft.ifft2(ehat).real
    eta *= (hs_frac * float(tb.get("hs", 0.5)) / 4.0) / max(eta.std(), 1e-300)
    ehat = np.fft.fft2(eta) * tb["aal"]
    y = np.zeros(6 * nx * ny)
    y[: nx * ny] = ehat.real.ravel()
    y[nx * ny: 2 * nx * ny] = ehat.imag.ravel()
    return y


def compare_2d(mlp, tb, t_warm=0.25, t_end=0.75, device=0, eps_abs=1e-8, eps_rel=1e-6, uniform=True):
    """The 2D learned variant beside the plain path on one varying-bottom deck: the
    plain 16-reference operator and the learned 4-reference blend (learned_tables2d),
    each from the same sea state over the whole domain (wave_field_2d) through t_warm
    and then, device-timed on the engine's own stream, to t_end; simulated seconds
    per wall second of each, RHS calls, and the eta relative L2 error of the learned
    run at t_end against the plain one (and, for scale, of uniform weights over the
    same 4 depths)."""
    import torch
    from . import decks2d
    from .engine2d import Engine2D
    n = tb["nx"] * tb["ny"]
    y0 = wave_field_2d(tb)
    lrn = learned_tables2d(mlp, tb)
    variants = [("plain", decks2d.plain_k_operator(tb, K_PLAIN)), ("learned", lrn)]
    if uniform:
        variants.append(("uniform", decks2d.with_k_operator(tb, lrn["ref_depths"],
                                                            np.full((K_LEARN,) + tb["depth"].shape, 1.0 / K_LEARN))))
    out, etas = {}, {}
    for name, t in variants:
        eng = Engine2D(t, eps_abs, eps_rel, device=device)
        st = torch.cuda.Stream(device=device)
        eng.set_stream(st.cuda_stream)
        eng.set_state(0.0, 0.02, y0)
        eng.run_to_time(t_warm)
        r0 = eng.stats()["rhs_calls"]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        eng.run_to_time(t_end)
        e1.record(st)
        torch.cuda.synchronize()
        if name != "uniform":
            out[f"{name}_sim_s_per_wall_s"] = (t_end - t_warm) / (e0.elapsed_time(e1) / 1e3)
            out[f"{name}_rhs_calls"] = eng.stats()["rhs_calls"] - r0
        etas[name] = eng.fields()[0]
        eng.close()
    err = lambda a: float(np.linalg.norm(a - etas["plain"]) / max(np.linalg.norm(etas["plain"]), 1e-300))
    out.update(speedup=out["learned_sim_s_per_wall_s"] / out["plain_sim_s_per_wall_s"],
               eta_err=err(etas["learned"]),
               eta_err_uniform_weights=err(etas["uniform"]) if "uniform" in etas else None,
               window_s=[t_warm, t_end])
    return out


def pipeline(n_train=512, n_eval=64, nx=16384, t_train=20.0, t_eval=20.0, epochs=200, batch=4096, stride=16,
             root=None, device=0, seed=0, log=print, save=None):
    """Config-4 pipeline: plain 16-reference runs on n_train random bathymetries ->
    training records -> GPU training -> a batched n_eval-member learned ensemble and
    the plain 16-reference ensemble on held-out bathymetries, both timed; returns the
    eta errors and the two ensembles' simulated-seconds per wall-second."""
    import os
    import tempfile
    import time
    from . import decks as _decks
    root = root or os.path.join(tempfile.gettempdir(), "hw_learned")
    tr = [_decks.config4_deck(os.path.join(root, f"train{i:04d}"), seed=seed + i, nx=nx, T_end=max(t_train, t_eval) + 10)
          for i in range(n_train)]
    ev = [_decks.config4_deck(os.path.join(root, f"eval{i:04d}"), seed=seed + 100000 + i, nx=nx,
                              T_end=max(t_train, t_eval) + 10) for i in range(n_eval)]
    log(f"{n_train} training and {n_eval} evaluation decks")
    t0 = time.time()
    recs = []
    for c in range(0, n_train, 64):
        recs.append(training_records(tr[c:c + 64], t_train, stride=stride, device=device))
    R = np.concatenate(recs)
    log(f"{R.shape[0]} training records from the plain runs in {time.time() - t0:.1f} s")
    mlp = MLP(seed=seed + 1, device=device)
    t0 = time.time()
    losses = train_staged(mlp, R, epochs=epochs, batch=batch)
    log(f"trained: loss {losses[0]:.3e} -> {losses[-1]:.3e} in {time.time() - t0:.1f} s")
    out = {"records": int(R.shape[0]), "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
           "n_train": n_train, "n_eval": n_eval}
    if save:
        np.save(save, mlp.params())
        log(f"network saved to {save}")

    def timed(eng):
        eng.run_to_time(0.5)
        s0 = sum(eng.state(m)[0] for m in range(eng.members))
        t = time.time()
        eng.run_to_time(t_eval)
        wall = time.time() - t
        s1 = sum(eng.state(m)[0] for m in range(eng.members))
        return (s1 - s0) / wall, wall

    plain = _eng.Engine(ev, eps_abs=1e-8, eps_rel=1e-6, nref=K_PLAIN, device=device)
    out["plain_sim_s_per_wall_s"], out["plain_wall_s"] = timed(plain)
    lrn = _eng.Engine(ev, eps_abs=1e-8, eps_rel=1e-6, nref=K_LEARN, device=device)
    install(lrn, ev, [learned_weights(mlp, d) for d in ev])
    out["learned_sim_s_per_wall_s"], out["learned_wall_s"] = timed(lrn)
    uni = _eng.Engine(ev, eps_abs=1e-8, eps_rel=1e-6, nref=K_LEARN, device=device)
    install(uni, ev, [(np.full((K_LEARN, n), 0.25), reference_depths(_eng.deck_table(d, "depth"), K_LEARN))
                      for d, n in zip(ev, uni.nx)])
    uni.run_to_time(t_eval)
    err_l, err_u = [], []
    for m in range(len(ev)):
        ep = eta_of(plain.state(m)[2], plain.nx[m])
        den = max(np.linalg.norm(ep), 1e-300)
        err_l.append(float(np.linalg.norm(eta_of(lrn.state(m)[2], lrn.nx[m]) - ep) / den))
        err_u.append(float(np.linalg.norm(eta_of(uni.state(m)[2], uni.nx[m]) - ep) / den))
    out.update(eta_err_learned_median=float(np.median(err_l)), eta_err_learned_max=float(np.max(err_l)),
               eta_err_uniform_median=float(np.median(err_u)),
               speedup=out["learned_sim_s_per_wall_s"] / out["plain_sim_s_per_wall_s"],
               rhs_calls_plain=sum(plain.stats(m)["rhs_calls"] for m in range(len(ev))),
               rhs_calls_learned=sum(lrn.stats(m)["rhs_calls"] for m in range(len(ev))))
    return out


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train and evaluate the learned K=4 depth operator")
    ap.add_argument("--train", type=int, default=512)
    ap.add_argument("--eval", type=int, default=64)
    ap.add_argument("--nx", type=int, default=16384)
    ap.add_argument("--t-train", type=float, default=20.0)
    ap.add_argument("--t-eval", type=float, default=20.0)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--stride", type=int, default=16)
    ap.add_argument("--save", default=None, help="write the trained network's parameters (.npy) here")
    a = ap.parse_args()
    res = pipeline(a.train, a.eval, a.nx, a.t_train, a.t_eval, a.epochs, stride=a.stride, save=a.save)
    print(json.dumps(res))
