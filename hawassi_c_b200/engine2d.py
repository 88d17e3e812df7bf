"""ctypes binding of the 2D entry points (hw2d_*) of include/hawassi_b200.h.

:class:`Engine2D` takes the operator tables of a 2D flat-bottom deck (the dict
built by :mod:`hawassi_c_b200.decks2d`, or the reference's own set-up globals)
and exposes ``rhs`` (rhs_AB2_2DF_uv, 2d/fun_odesolver.c:4458), ``evolve_apply``
(gsl_odeiv2_evolve_apply, :2643) and ``run_to_time`` (the inner loop of
ode_solver_uv, :2641-2647) with the state resident on the device.
"""
import ctypes
import os

import numpy as np

from .engine import EngineError, HwOpts, load_library

_dp = ctypes.POINTER(ctypes.c_double)


class Hw2dTables(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("model", ctypes.c_int), ("propagation", ctypes.c_int),
        ("cpeak", ctypes.c_double),
        ("kx", _dp), ("ky", _dp), ("c2d", _dp), ("l2d", _dp), ("aal", _dp), ("charac", _dp), ("chiadj", _dp),
        ("newgam", _dp), ("skewgam", _dp),
        ("nt", ctypes.c_int), ("tsig", _dp), ("sig", _dp), ("sigskew", _dp),
        ("gam_min", _dp), ("gam_plus", _dp), ("csq_min", _dp), ("csq_plus", _dp), ("om2_min", _dp),
        ("om2_plus", _dp), ("wallchar", _dp),
        ("breaking", ctypes.c_int), ("bathy", _dp), ("brchar", _dp), ("x", _dp), ("y", _dp),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("max_eta_init", ctypes.c_double),
        ("tstar", ctypes.c_double), ("rsearch", ctypes.c_double), ("kbc", ctypes.c_double), ("tc", ctypes.c_double),
        ("delb", ctypes.c_double), ("cur_u", ctypes.c_double), ("t0", ctypes.c_double), ("dt_out", ctypes.c_double),
        ("refl_coef", ctypes.c_double),
        ("gam_mid", _dp), ("csq_mid", _dp), ("om2_mid", _dp),
        ("nrefk", ctypes.c_int), ("gam_k", _dp), ("csq_k", _dp), ("om2_k", _dp),
    ]


class Hw2dOutputs(ctypes.Structure):
    _fields_ = [
        ("outdir", ctypes.c_char_p), ("nt", ctypes.c_int), ("tout", _dp), ("dt", ctypes.c_double),
        ("npartition", ctypes.c_int), ("uv_every_sample", ctypes.c_int),
        ("hs", ctypes.c_double), ("kp", ctypes.c_double), ("wp", ctypes.c_double),
        ("x", _dp), ("y", _dp), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("kx", _dp), ("ky", _dp), ("bathy", _dp), ("cfsa", _dp), ("chiadjphi", _dp),
        ("ngauge", ctypes.c_int), ("xgauge", _dp), ("ygauge", _dp),
    ]


def output_spec(struct, outdir, tout, dt, npartition, x, y, dx, dy, kx, ky, bathy, cfsa, chiadjphi=None,
                hs=0.0, kp=0.0, wp=0.0, gauges=None, uv_every_sample=False):
    """Fill an outputs structure (hw2d_outputs layout); returns it and the arrays it
    points into, which the caller keeps alive for the call."""
    keep = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in
            dict(tout=tout, x=x, y=y, kx=kx, ky=ky, bathy=bathy, cfsa=cfsa).items()}
    keep["chiadjphi"] = None if chiadjphi is None else np.ascontiguousarray(chiadjphi, dtype=np.float64)
    g = np.zeros((0, 2)) if gauges is None else np.asarray(gauges, dtype=np.float64).reshape(-1, 2)
    keep["xgauge"], keep["ygauge"] = np.ascontiguousarray(g[:, 0]), np.ascontiguousarray(g[:, 1])
    keep["outdir"] = os.path.join(str(outdir), "").encode()
    spec = struct(outdir=keep["outdir"], nt=len(keep["tout"]), dt=float(dt), npartition=int(npartition),
                  uv_every_sample=int(bool(uv_every_sample)), hs=float(hs), kp=float(kp), wp=float(wp),
                  dx=float(dx), dy=float(dy), ngauge=len(g),
                  **{k: _ptr(keep[k]) if len(g) or k not in ("xgauge", "ygauge") else None
                     for k in ("tout", "x", "y", "kx", "ky", "bathy", "cfsa", "chiadjphi", "xgauge", "ygauge")})
    return spec, keep


# parambreak's scalars (2d/breaking.c:1-8) as the tables dict carries them
BREAKING_SCALARS = ("dx", "dy", "max_eta_init", "tstar", "rsearch", "kbc", "tc", "delb", "cur_u", "t0", "dt_out")


_bound = False


def _lib():
    global _bound
    L = load_library()
    if not _bound:
        vp, dp, dd = ctypes.c_void_p, _dp, ctypes.c_double
        llp = ctypes.POINTER(ctypes.c_longlong)
        L.hw2d_create.restype = vp
        L.hw2d_create.argtypes = [ctypes.POINTER(Hw2dTables), ctypes.POINTER(HwOpts)]
        L.hw2d_destroy.argtypes = [vp]
        L.hw2d_last_error.restype = ctypes.c_char_p
        L.hw2d_last_error.argtypes = [vp]
        L.hw2d_nx.argtypes = [vp]
        L.hw2d_ny.argtypes = [vp]
        L.hw2d_rhs.argtypes = [vp, dd, dp, dp]
        L.hw2d_gsl_rhs.argtypes = [dd, dp, dp, vp]
        L.hw2d_evolve_apply.argtypes = [vp, dp, dd, dp, dp]
        L.hw2d_set_state.argtypes = [vp, dd, dd, dp]
        L.hw2d_get_state.argtypes = [vp, dp, dp, dp]
        L.hw2d_run_to_time.argtypes = [vp, dd]
        L.hw2d_stats.argtypes = [vp, llp, llp, llp]
        L.hw2d_set_stream.argtypes = [vp, vp]
        L.hw2d_synchronize.argtypes = [vp]
        L.hw2d_launches.restype = ctypes.c_longlong
        L.hw2d_launches.argtypes = [vp]
        ip = ctypes.POINTER(ctypes.c_int)
        L.hw2d_breaking_fields.argtypes = [vp, dp, dp, dp, ip, ip]
        L.hw2d_breaking_log.argtypes = [vp, dp, ip, ip, ctypes.c_int, ctypes.c_longlong]
        L.hw2d_breaking_log_nodes.restype = ctypes.c_longlong
        L.hw2d_breaking_log_nodes.argtypes = [vp]
        L.hw2d_fields.argtypes = [vp, dp, dp, dp]
        L.hw2d_run_outputs.argtypes = [vp, ctypes.POINTER(Hw2dOutputs)]
        L.hw2d_directional_influx.argtypes = [ctypes.c_int, dd, dd, ctypes.c_int, dp, dd, ctypes.c_int, dp, dp, dp,
                                              dp, dp, dd, dp, dp, dp, dp, ctypes.c_int]
        L.hw2d_influx_last_error.restype = ctypes.c_char_p
        _bound = True
    return L


def directional_signal(t0, dt, nt, y, y0, comps, mdir=0.0, ramp_t=None, ramp_y=None, device=0):
    """The directional line signal and its quadrature ([lines][nt] each) of the
    components comps = (a, w, k, theta, phi) on the device (hw2d_directional_influx)."""
    L = _lib()
    y = np.ascontiguousarray(y, dtype=np.float64)
    a, w, k, th, ph = (np.ascontiguousarray(v, dtype=np.float64) for v in comps)
    rt = np.ones(nt) if ramp_t is None else np.ascontiguousarray(ramp_t, dtype=np.float64)
    ry = np.ones(y.size) if ramp_y is None else np.ascontiguousarray(ramp_y, dtype=np.float64)
    eta, skew = np.empty((y.size, nt)), np.empty((y.size, nt))
    if L.hw2d_directional_influx(int(nt), float(t0), float(dt), y.size, _ptr(y), float(y0), a.size, _ptr(a), _ptr(w),
                                 _ptr(k), _ptr(th), _ptr(ph), float(mdir), _ptr(rt), _ptr(ry), _ptr(eta), _ptr(skew),
                                 int(device)):
        raise EngineError(L.hw2d_influx_last_error().decode())
    return eta, skew


def _ptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


class Engine2D:
    def __init__(self, tables, eps_abs=0.0, eps_rel=0.0, h0=0.0, device=0):
        self._L = _lib()
        keep = {}
        for k in ("kx", "ky", "c2d", "l2d", "aal", "charac", "chiadj", "newgam", "skewgam", "tsig", "sig", "sigskew",
                  "gam_min", "gam_plus", "csq_min", "csq_plus", "om2_min", "om2_plus", "wallchar", "gam_mid",
                  "csq_mid", "om2_mid", "gam_k", "csq_k", "om2_k"):
            v = tables.get(k)
            keep[k] = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        brk = int(tables.get("breaking", 0))
        for k in ("bathy", "brchar", "x", "y"):
            keep[k] = np.ascontiguousarray(tables[k], dtype=np.float64) if brk else None
        self._keep = keep
        scal = {k: float(tables.get(k, 0.0)) for k in BREAKING_SCALARS}
        tb = Hw2dTables(nx=int(tables["nx"]), ny=int(tables["ny"]), model=int(tables.get("model", 2)),
                        propagation=int(tables.get("propagation", 0)), cpeak=float(tables["cpeak"]),
                        nt=int(tables.get("nt", 0) if keep["sig"] is not None else 0), breaking=brk, **scal,
                        refl_coef=float(tables.get("refl_coef", 0.0)), nrefk=int(tables.get("nrefk", 0)),
                        **{k: _ptr(v) for k, v in keep.items()})
        o = HwOpts(eps_abs=eps_abs, eps_rel=eps_rel, h0=h0, device=device)
        self._h = self._L.hw2d_create(ctypes.byref(tb), ctypes.byref(o))
        if not self._h:
            raise EngineError(self._L.hw2d_last_error(None).decode())
        self.nx, self.ny = int(tables["nx"]), int(tables["ny"])
        self.n = self.nx * self.ny

    def _err(self):
        return EngineError(self._L.hw2d_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.hw2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rhs(self, t, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.empty(6 * self.n)
        if self._L.hw2d_rhs(self._h, float(t), _ptr(y), _ptr(out)):
            raise self._err()
        return out

    def evolve_apply(self, t, t1, h, y):
        """One gsl_odeiv2_evolve_apply call; y (float64, 6*nx*ny) is updated in place."""
        tt, hh = ctypes.c_double(t), ctypes.c_double(h)
        if self._L.hw2d_evolve_apply(self._h, ctypes.byref(tt), float(t1), ctypes.byref(hh), _ptr(y)):
            raise self._err()
        return tt.value, hh.value

    def set_state(self, t, h, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        if self._L.hw2d_set_state(self._h, float(t), float(h), _ptr(y)):
            raise self._err()

    def state(self, with_y=True):
        t, h = ctypes.c_double(), ctypes.c_double()
        y = np.empty(6 * self.n) if with_y else None
        if self._L.hw2d_get_state(self._h, ctypes.byref(t), ctypes.byref(h), _ptr(y)):
            raise self._err()
        return t.value, h.value, y

    def state_into(self, y):
        """Read the state into the caller's float64 array (pinned memory makes the copy
        a direct DMA); returns (t, h)."""
        t, h = ctypes.c_double(), ctypes.c_double()
        if self._L.hw2d_get_state(self._h, ctypes.byref(t), ctypes.byref(h), _ptr(y)):
            raise self._err()
        return t.value, h.value

    def run_to_time(self, t1):
        if self._L.hw2d_run_to_time(self._h, float(t1)):
            raise self._err()

    def stats(self):
        r, a, j = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        if self._L.hw2d_stats(self._h, ctypes.byref(r), ctypes.byref(a), ctypes.byref(j)):
            raise self._err()
        return {"rhs_calls": r.value, "accepted": a.value, "rejected": j.value}

    def set_stream(self, stream_handle):
        if self._L.hw2d_set_stream(self._h, ctypes.c_void_p(stream_handle)):
            raise self._err()

    def launches(self):
        return int(self._L.hw2d_launches(self._h))

    def synchronize(self):
        if self._L.hw2d_synchronize(self._h):
            raise self._err()

    def breaking_fields(self):
        """B, Sb_xhat, Sb_yhat (complex [ny, nx]), flagbr and the tracked crests after
        the last RHS (the globals of 2d/breaking.c)."""
        n = self.nx * self.ny
        B = np.zeros(n)
        sx, sy = np.zeros(2 * n), np.zeros(2 * n)
        fl, nc = ctypes.c_int(), ctypes.c_int()
        if self._L.hw2d_breaking_fields(self._h, _ptr(B), _ptr(sx), _ptr(sy), ctypes.byref(fl), ctypes.byref(nc)):
            raise self._err()
        shp = (self.ny, self.nx)
        return (B.reshape(shp), (sx[0::2] + 1j * sx[1::2]).reshape(shp), (sy[0::2] + 1j * sy[1::2]).reshape(shp),
                fl.value, nc.value)

    def breaking_log(self):
        """breaking.dat records as a list of (t, [(x index, y index), ...])."""
        L = self._L
        nn = int(L.hw2d_breaking_log_nodes(self._h))
        nr = L.hw2d_breaking_log(self._h, None, None, None, 0, 0)
        if nr < 0:
            raise EngineError("hw2d_breaking_log: " + ("log overflow" if nr == -2 else "no breaking"))
        t = np.zeros(max(nr, 1))
        cnt = np.zeros(max(nr, 1), dtype=np.int32)
        nodes = np.zeros(2 * max(nn, 1), dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        L.hw2d_breaking_log(self._h, _ptr(t), cnt.ctypes.data_as(ip), nodes.ctypes.data_as(ip), nr, nn)
        out, off = [], 0
        for r in range(nr):
            c = int(cnt[r])
            out.append((float(t[r]), [tuple(v) for v in nodes[2 * off:2 * (off + c)].reshape(-1, 2).tolist()]))
            off += c
        return out

    def fields(self):
        """eta, u, v ([ny, nx] each) of the device state: ifftw_2d_c2r of each spectrum
        (2d/functions1.c:523-557), as ode_solver_uv forms them at an output time."""
        out = [np.empty(self.n) for _ in range(3)]
        if self._L.hw2d_fields(self._h, *[_ptr(a) for a in out]):
            raise self._err()
        return tuple(a.reshape(self.ny, self.nx) for a in out)

    def run_outputs(self, outdir, tout, dt, npartition, x, y, dx, dy, kx, ky, bathy, cfsa, chiadjphi=None,
                    hs=0.0, kp=0.0, wp=0.0, gauges=None, uv_every_sample=False):
        """ode_solver_uv's time loop with its output files (hw2d_run_outputs) from the
        device state; gauges is a sequence of (x, y) as gauges.dat lists them.
        Returns the samples written."""
        spec, keep = output_spec(Hw2dOutputs, outdir, tout, dt, npartition, x, y, dx, dy, kx, ky, bathy, cfsa,
                                 chiadjphi, hs, kp, wp, gauges, uv_every_sample)
        r = self._L.hw2d_run_outputs(self._h, ctypes.byref(spec))
        del keep
        if r < 0:
            raise self._err()
        return r
