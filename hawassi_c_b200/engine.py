"""ctypes binding of the C ABI in include/hawassi_b200.h."""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libhawassi_b200.so")
_lib = None


class EngineError(RuntimeError):
    pass


class HwOpts(ctypes.Structure):
    _fields_ = [
        ("eps_abs", ctypes.c_double),
        ("eps_rel", ctypes.c_double),
        ("h0", ctypes.c_double),
        ("seed", ctypes.c_ulonglong),
        ("nref", ctypes.c_int),
        ("exact_sequence", ctypes.c_int),
        ("cluster", ctypes.c_int),
        ("device", ctypes.c_int),
        ("slice", ctypes.c_int),
        ("resident", ctypes.c_int),
    ]


def library_path():
    return _LIB_PATH


EXPORTS = [
    "hw_create", "hw_ensemble_create", "hw_ensemble_create_sliced", "hw_destroy", "hw_last_error", "hw_members", "hw_nx", "hw_nt",
    "hw_initial_state", "hw_rhs", "hw_gsl_rhs", "hw_evolve_apply", "hw_run", "hw_run_to_time",
    "hw_get_state", "hw_set_state", "hw_reset", "hw_member_stats", "hw_last_dydt", "hw_breaking_log",
    "hw_set_stream", "hw_synchronize", "hw_deck_table", "hw_get_states", "hw_set_states",
    "hw_class_timing", "hw_rhs_noalloc", "hw_energy", "hw_run_members", "hw_set_operator_weights",
    "hw_mlp_sizes", "hw_mlp_create", "hw_mlp_destroy", "hw_mlp_last_error", "hw_mlp_get_params",
    "hw_mlp_set_params", "hw_mlp_grad", "hw_mlp_grad_device", "hw_mlp_train", "hw_mlp_infer",
    "hw2d_create", "hw2d_destroy", "hw2d_last_error", "hw2d_nx", "hw2d_ny", "hw2d_rhs", "hw2d_gsl_rhs",
    "hw2d_evolve_apply", "hw2d_set_state", "hw2d_get_state", "hw2d_run_to_time", "hw2d_stats",
    "hw2d_set_stream", "hw2d_synchronize", "hw2d_launches", "hw_gauges", "hw_ngauge", "hw_enable_fields", "hw_write_outputs",
]


def load_library():
    """Load the CUDA engine; raises EngineError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise EngineError(f"CUDA engine not built: {_LIB_PATH} is missing (python -m hawassi_c_b200.build)")
    L = ctypes.CDLL(_LIB_PATH)
    vp, dp, ip, dd = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_double
    llp = ctypes.POINTER(ctypes.c_longlong)
    L.hw_create.restype = vp
    L.hw_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(HwOpts)]
    L.hw_ensemble_create.restype = vp
    L.hw_ensemble_create.argtypes = [ctypes.POINTER(ctypes.c_char_p), ip, ctypes.POINTER(HwOpts)]
    L.hw_ensemble_create_sliced.restype = vp
    L.hw_ensemble_create_sliced.argtypes = [ctypes.POINTER(ctypes.c_char_p), ip, ctypes.POINTER(HwOpts),
                                            ctypes.POINTER(ctypes.c_int)]
    L.hw_destroy.argtypes = [vp]
    L.hw_last_error.restype = ctypes.c_char_p
    L.hw_last_error.argtypes = [vp]
    L.hw_members.argtypes = [vp]
    L.hw_nx.argtypes = [vp, ip]
    L.hw_nt.argtypes = [vp, ip]
    L.hw_initial_state.argtypes = [vp, ip, dp]
    L.hw_rhs.argtypes = [vp, ip, dd, dp, dp]
    L.hw_gsl_rhs.argtypes = [dd, dp, dp, vp]
    L.hw_evolve_apply.argtypes = [vp, ip, dp, dd, dp, dp]
    L.hw_run.argtypes = [vp, ip]
    L.hw_run_to_time.argtypes = [vp, dd]
    L.hw_get_state.argtypes = [vp, ip, dp, dp, dp]
    L.hw_set_state.argtypes = [vp, ip, dd, dd, dp, ip]
    L.hw_reset.argtypes = [vp]
    L.hw_member_stats.argtypes = [vp, ip, llp, llp, llp, ctypes.POINTER(ctypes.c_int)]
    L.hw_last_dydt.argtypes = [vp, ip, dp]
    L.hw_breaking_log.argtypes = [vp, ip, dp, ctypes.c_longlong, llp]
    L.hw_set_stream.argtypes = [vp, vp]
    L.hw_synchronize.argtypes = [vp]
    L.hw_deck_table.argtypes = [ctypes.c_char_p, ctypes.POINTER(HwOpts), ctypes.c_char_p, dp, ip]
    L.hw_rhs_noalloc.argtypes = [vp, ip, dd, vp, vp, vp]
    L.hw_gauges.argtypes = [vp, ip, dp, dp, dp, ip]
    L.hw_kinematics_dims.argtypes = [vp, ip, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.hw_kinematics_grid.argtypes = [vp, ip, dp, dp]
    L.hw_kinematics.argtypes = [vp, ip, dd, dp, dp, dp, dp, dp, dp]
    L.hw_ngauge.argtypes = [vp, ip]
    L.hw_enable_fields.argtypes = [vp, ip, ip]
    L.hw_write_outputs.argtypes = [vp, ip, ctypes.c_char_p]
    L.hw_energy.argtypes = [vp, ip, dp, dp]
    L.hw_run_members.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.hw_set_operator_weights.argtypes = [vp, ip, ip, dp, dp]
    fp = ctypes.POINTER(ctypes.c_float)
    ipp = ctypes.POINTER(ctypes.c_int)
    L.hw_mlp_sizes.argtypes = [ipp, ipp, ipp, ipp, ipp]
    L.hw_mlp_create.restype = vp
    L.hw_mlp_create.argtypes = [ctypes.c_ulonglong, ip]
    L.hw_mlp_destroy.argtypes = [vp]
    L.hw_mlp_last_error.restype = ctypes.c_char_p
    L.hw_mlp_last_error.argtypes = [vp]
    L.hw_mlp_get_params.argtypes = [vp, fp]
    L.hw_mlp_set_params.argtypes = [vp, fp]
    L.hw_mlp_grad.argtypes = [vp, fp, ip, fp, fp]
    L.hw_mlp_grad_device.argtypes = [vp, vp, ip, fp, fp]
    L.hw_mlp_train.argtypes = [vp, fp, ip, ip, ip, ctypes.c_float, fp]
    L.hw_mlp_infer.argtypes = [vp, fp, ip, dp]
    L.hw_get_states.argtypes = [vp, dp]
    L.hw_set_states.argtypes = [vp, dp]
    L.hw_class_timing.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ip]
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Engine:
    """One deck directory (``Engine("deck")``) or a ragged ensemble
    (``Engine(["deck0", "deck1", ...])``) on one GPU."""

    def __init__(self, decks, eps_abs=0.0, eps_rel=0.0, h0=0.0, seed=0, nref=0, exact_sequence=False,
                 cluster=0, device=0, slice=0, slices=None, resident=0):
        """slices: grid points per CTA per grid size ({Nx: points}, e.g. from
        autotune.autotune_slices) or per member (a list); others use `slice`.
        resident: the evolve launches' grid (hw_opts.resident): 0 one cluster per
        member, -1 a persistent grid of resident clusters pulling members from a
        queue (sized to the class's share), n > 0 at most n such clusters per class."""
        L = load_library()
        if isinstance(decks, (str, os.PathLike)):
            decks = [decks]
        self.decks = [os.fspath(d) for d in decks]
        opts = HwOpts(eps_abs, eps_rel, h0, seed, nref, int(bool(exact_sequence)), cluster, device, slice,
                      int(resident))
        arr = (ctypes.c_char_p * len(self.decks))(*[d.encode() for d in self.decks])
        if slices is None:
            self._h = L.hw_ensemble_create(arr, len(self.decks), ctypes.byref(opts))
        else:
            if isinstance(slices, dict):
                per = [int(slices.get(int(deck_table(d, "Nx")[0]), 0)) for d in self.decks]
            else:
                per = [int(v) for v in slices]
            ms = (ctypes.c_int * len(self.decks))(*per)
            self._h = L.hw_ensemble_create_sliced(arr, len(self.decks), ctypes.byref(opts), ms)
        if not self._h:
            raise EngineError(L.hw_last_error(None).decode())
        self.members = L.hw_members(self._h)
        self.nx = [L.hw_nx(self._h, i) for i in range(self.members)]
        self.nt = [L.hw_nt(self._h, i) for i in range(self.members)]

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            load_library().hw_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc, what):
        if rc != 0:
            raise EngineError(f"{what}: " + load_library().hw_last_error(self._h).decode())

    # -- reference call surface ----------------------------------------------
    def initial_state(self, member=0):
        y = np.zeros(4 * self.nx[member])
        self._check(load_library().hw_initial_state(self._h, member, _dp(y)), "initial_state")
        return y

    def rhs(self, t, y, member=0):
        y = np.ascontiguousarray(y, dtype=np.float64)
        dz = np.empty_like(y)
        self._check(load_library().hw_rhs(self._h, member, float(t), _dp(y), _dp(dz)), "rhs")
        return dz

    def rhs_noalloc(self, t, y_dev_ptr, dydt_dev_ptr, stream=0, member=0):
        """RHS on caller-owned device buffers (reference layout) with no device
        allocation at call time; asynchronous on `stream` (a cudaStream_t value)."""
        rc = load_library().hw_rhs_noalloc(self._h, member, float(t), ctypes.c_void_p(y_dev_ptr),
                                           ctypes.c_void_p(dydt_dev_ptr), ctypes.c_void_p(stream))
        self._check(rc, "rhs_noalloc")

    def evolve_apply(self, t, t1, h, y, member=0):
        """In place on y; returns (t, h) like gsl_odeiv_evolve_apply's outputs."""
        tt = np.array([t], dtype=np.float64)
        hh = np.array([h], dtype=np.float64)
        rc = load_library().hw_evolve_apply(self._h, member, _dp(tt), float(t1), _dp(hh), _dp(y))
        self._check(rc, "evolve_apply")
        return float(tt[0]), float(hh[0])

    def run(self, i_stop=-1, sync=True):
        self._check(load_library().hw_run(self._h, int(i_stop)), "run")
        if sync:
            self.synchronize()

    def run_members(self, i_stop, sync=True):
        """Advance each member m through output sample i_stop[m] (exclusive); members
        whose stop is not past their current index hold."""
        arr = (ctypes.c_int * self.members)(*[int(v) for v in i_stop])
        self._check(load_library().hw_run_members(self._h, arr), "run_members")
        if sync:
            self.synchronize()

    def set_operator_weights(self, member, depths, gam):
        """Install K reference depths and per-point weights gam[K][Nx] (varying-depth member)."""
        d = np.ascontiguousarray(depths, dtype=np.float64)
        g = np.ascontiguousarray(gam, dtype=np.float64)
        self._check(load_library().hw_set_operator_weights(self._h, member, d.size, _dp(d), _dp(g)),
                    "set_operator_weights")

    def run_to_time(self, t_end, sync=True):
        self._check(load_library().hw_run_to_time(self._h, float(t_end)), "run_to_time")
        if sync:
            self.synchronize()

    def state(self, member=0):
        y = np.zeros(4 * self.nx[member])
        t = np.zeros(1)
        h = np.zeros(1)
        self._check(load_library().hw_get_state(self._h, member, _dp(t), _dp(h), _dp(y)), "get_state")
        return float(t[0]), float(h[0]), y

    def set_state(self, t, h, y, member=0, i_out=0):
        y = np.ascontiguousarray(y, dtype=np.float64) if y is not None else None
        rc = load_library().hw_set_state(self._h, member, float(t), float(h),
                                         _dp(y) if y is not None else None, int(i_out))
        self._check(rc, "set_state")

    def reset(self):
        self._check(load_library().hw_reset(self._h), "reset")

    def stats(self, member=0):
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        s = ctypes.c_int()
        self._check(load_library().hw_member_stats(self._h, member, ctypes.byref(a), ctypes.byref(b),
                                                   ctypes.byref(c), ctypes.byref(s)), "stats")
        return {"rhs_calls": a.value, "accepted": b.value, "rejected": c.value, "status": s.value}

    def energy(self, y=None, member=0):
        """Quadratic Hamiltonian of y (host state) or of the member's current state."""
        e = np.zeros(1)
        yy = None if y is None else np.ascontiguousarray(y, dtype=np.float64)
        self._check(load_library().hw_energy(self._h, member, _dp(yy) if yy is not None else None, _dp(e)),
                    "energy")
        return float(e[0])

    def last_dydt(self, member=0):
        y = np.zeros(4 * self.nx[member])
        self._check(load_library().hw_last_dydt(self._h, member, _dp(y)), "last_dydt")
        return y

    def kinematics(self, tprev, member=0):
        """kinematic_modul at the member's current time (deck with kinematic yes): dict of
        eta_cut [nx_out], P, dxphi, dzphi, dtdxphi, dtdzphi [nx_out, nz_out], x_out, z_out."""
        L = load_library()
        a, b = ctypes.c_int(), ctypes.c_int()
        self._check(L.hw_kinematics_dims(self._h, member, ctypes.byref(a), ctypes.byref(b)), "hw_kinematics_dims")
        nxo, nz = a.value, b.value
        xo, zo = np.zeros(nxo), np.zeros(nz)
        self._check(L.hw_kinematics_grid(self._h, member, _dp(xo), _dp(zo)), "hw_kinematics_grid")
        out = {k: np.zeros(nxo * nz) for k in ("P", "dxphi", "dzphi", "dtdxphi", "dtdzphi")}
        ec = np.zeros(nxo)
        self._check(L.hw_kinematics(self._h, member, float(tprev), _dp(ec), _dp(out["P"]), _dp(out["dxphi"]),
                                    _dp(out["dzphi"]), _dp(out["dtdxphi"]), _dp(out["dtdzphi"])), "hw_kinematics")
        res = {k: v.reshape(nxo, nz) for k, v in out.items()}
        res.update(eta_cut=ec, x_out=xo, z_out=zo)
        return res

    def gauges(self, member=0):
        """Gauge series the device computed at every output sample reached so far:
        (tim [rows], eta [rows, ngauge], deta/dt [rows, ngauge])."""
        L = load_library()
        ng = L.hw_ngauge(self._h, member)
        cap = max(self.nt[member] if hasattr(self, "nt") else 0, 1)
        cap = max(cap, L.hw_nt(self._h, member))
        eta = np.zeros((cap, max(ng, 1)))
        dt = np.zeros((cap, max(ng, 1)))
        tim = np.zeros(cap)
        rows = L.hw_gauges(self._h, member, _dp(eta), _dp(dt), _dp(tim), cap)
        if rows < 0:
            raise EngineError(L.hw_last_error(self._h).decode())
        return tim[:rows], eta[:rows, :ng], dt[:rows, :ng]

    def enable_fields(self, member=0, enable=True):
        """Keep eta, u, phi of every output sample of the member on the device."""
        self._check(load_library().hw_enable_fields(self._h, member, int(bool(enable))), "enable_fields")

    def write_outputs(self, outdir, member=0):
        """The reference's output files (Constants/Hawassi_*_NN.dat, gauge text files,
        breaking.dat) of the member into outdir; returns the samples written."""
        import os
        os.makedirs(outdir, exist_ok=True)
        L = load_library()
        rows = L.hw_write_outputs(self._h, member, str(outdir).encode())
        if rows < 0:
            raise EngineError(L.hw_last_error(self._h).decode())
        return rows

    def breaking_log(self, member=0):
        """breaking.dat records [(t, [nodes...]), ...] of the member."""
        L = load_library()
        n = ctypes.c_longlong()
        if L.hw_breaking_log(self._h, member, None, 0, ctypes.byref(n)) < 0:
            raise EngineError(L.hw_last_error(self._h).decode())
        buf = np.zeros(max(n.value, 1))
        L.hw_breaking_log(self._h, member, _dp(buf), n.value, ctypes.byref(n))
        out, i = [], 0
        while i < n.value:
            t, cnt = buf[i], int(buf[i + 1])
            out.append((t, [int(v) for v in buf[i + 2:i + 2 + cnt]]))
            i += 2 + cnt
        return out

    def get_states(self, out):
        """All member states into one host buffer (concatenated reference layouts)."""
        self._check(load_library().hw_get_states(self._h, _dp(out)), "get_states")
        return out

    def set_states(self, y_all):
        """All member states from one host buffer (concatenated reference layouts).
        The copy is queued on the engine's stream: a pinned buffer must stay
        unchanged until the next synchronising call (run(sync=True), get_states)."""
        y_all = np.ascontiguousarray(y_all, dtype=np.float64)
        self._check(load_library().hw_set_states(self._h, _dp(y_all)), "set_states")

    def class_timing(self):
        """[(ms, members, grid_n), ...] of the last run's evolve launches."""
        L = load_library()
        ms = np.zeros(16)
        mem = (ctypes.c_int * 16)()
        gn = (ctypes.c_int * 16)()
        n = L.hw_class_timing(self._h, _dp(ms), mem, gn, 16)
        if n < 0:
            raise EngineError("class_timing failed")
        return [(float(ms[i]), int(mem[i]), int(gn[i])) for i in range(n)]

    def set_stream(self, stream_ptr):
        self._check(load_library().hw_set_stream(self._h, ctypes.c_void_p(stream_ptr)), "set_stream")

    def synchronize(self):
        self._check(load_library().hw_synchronize(self._h), "synchronize")


class HwJonswap(ctypes.Structure):
    _fields_ = [("T0", ctypes.c_double), ("Tend", ctypes.c_double), ("dt", ctypes.c_double),
                ("Tp", ctypes.c_double), ("Hs", ctypes.c_double), ("gamma", ctypes.c_double),
                ("nTramp", ctypes.c_double), ("seed", ctypes.c_ulonglong)]


def fp64_peak_tflops(device=0):
    """FP64 FMA throughput of the device in TFLOP/s (hw_fp64_peak_tflops)."""
    L = load_library()
    L.hw_fp64_peak_tflops.restype = ctypes.c_double
    L.hw_fp64_peak_tflops.argtypes = [ctypes.c_int]
    v = float(L.hw_fp64_peak_tflops(int(device)))
    if not v > 0:
        raise EngineError("hw_fp64_peak_tflops failed")
    return v


def jonswap_influx(specs, device=0):
    """Seeded JONSWAP influx signals of many members in one device launch
    (hw_jonswap_influx).  specs: dicts with T0, Tend, dt, Tp, Hs, gamma, nTramp, seed.
    Returns one array per member (samples at T0 + j dt)."""
    L = load_library()
    if not getattr(L, "_js_bound", False):
        L.hw_jonswap_influx.restype = ctypes.c_int
        L.hw_jonswap_influx.argtypes = [ctypes.POINTER(HwJonswap), ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                        ctypes.c_longlong, ctypes.c_int]
        L._js_bound = True
    arr = (HwJonswap * len(specs))(*[HwJonswap(**{k: (int(v) if k == "seed" else float(v)) for k, v in sp.items()})
                                    for sp in specs])
    total = L.hw_jonswap_influx(arr, len(specs), None, 0, device)
    if total < 0:
        raise EngineError("hw_jonswap_influx: invalid specification")
    out = np.zeros(total)
    if L.hw_jonswap_influx(arr, len(specs), _dp(out), total, device) != total:
        raise EngineError("hw_jonswap_influx failed")
    res, off = [], 0
    for sp in specs:
        nt = int((sp["Tend"] - sp["T0"]) / sp["dt"] + 1)
        res.append(out[off:off + nt])
        off += nt
    return res


def deck_table(deck, name, seed=0, nref=0):
    """Host-side set-up table of a deck (no GPU involved)."""
    L = load_library()
    opts = HwOpts(0.0, 0.0, 0.0, seed, nref, 0, 0, 0, 0, 0)
    n = L.hw_deck_table(os.fspath(deck).encode(), ctypes.byref(opts), name.encode(), None, 0)
    if n < 0:
        raise EngineError(L.hw_last_error(None).decode())
    out = np.zeros(max(n, 1))
    L.hw_deck_table(os.fspath(deck).encode(), ctypes.byref(opts), name.encode(), _dp(out), n)
    return out[:n]
