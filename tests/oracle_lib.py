"""ctypes wrapper around the CPU oracle (oracle/build/libhw_oracle.so).

Test infrastructure: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "build", "libhw_oracle.so")

_lib = None


class OrOpts(ctypes.Structure):
    _fields_ = [
        ("eps_abs", ctypes.c_double),
        ("eps_rel", ctypes.c_double),
        ("h0", ctypes.c_double),
        ("t_stop", ctypes.c_double),
        ("seed", ctypes.c_ulonglong),
        ("nref", ctypes.c_int),
        ("write_fields", ctypes.c_int),
        ("outdir", ctypes.c_char_p),
    ]


_dpt = ctypes.POINTER(ctypes.c_double)


class Or2dTables(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("model", ctypes.c_int), ("propagation", ctypes.c_int),
        ("cpeak", ctypes.c_double),
        ("kx", _dpt), ("ky", _dpt), ("c2d", _dpt), ("l2d", _dpt), ("aal", _dpt), ("charac", _dpt),
        ("chiadj", _dpt), ("newgam", _dpt), ("skewgam", _dpt),
        ("nt", ctypes.c_int), ("tsig", _dpt), ("sig", _dpt), ("sigskew", _dpt),
        ("gam_min", _dpt), ("gam_plus", _dpt), ("csq_min", _dpt), ("csq_plus", _dpt), ("om2_min", _dpt),
        ("om2_plus", _dpt), ("wallchar", _dpt),
        ("breaking", ctypes.c_int), ("bathy", _dpt), ("brchar", _dpt), ("x", _dpt), ("y", _dpt),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("max_eta_init", ctypes.c_double),
        ("tstar", ctypes.c_double), ("rsearch", ctypes.c_double), ("kbc", ctypes.c_double), ("tc", ctypes.c_double),
        ("delb", ctypes.c_double), ("cur_u", ctypes.c_double), ("t0", ctypes.c_double), ("dt_out", ctypes.c_double),
        ("refl_coef", ctypes.c_double),
        ("gam_mid", _dpt), ("csq_mid", _dpt), ("om2_mid", _dpt),
        ("nrefk", ctypes.c_int), ("gam_k", _dpt), ("csq_k", _dpt), ("om2_k", _dpt),
    ]

BRK_SCALARS = ("dx", "dy", "max_eta_init", "tstar", "rsearch", "kbc", "tc", "delb", "cur_u", "t0", "dt_out")


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        build()   # make: rebuilds only what changed
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
        L.or_create.restype = vp
        L.or_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(OrOpts)]
        L.or_destroy.argtypes = [vp]
        L.or_last_error.restype = ctypes.c_char_p
        L.or_nx.argtypes = [vp]
        L.or_nt.argtypes = [vp]
        L.or_scalar.restype = ctypes.c_double
        L.or_scalar.argtypes = [vp, ctypes.c_char_p]
        L.or_table.argtypes = [vp, ctypes.c_char_p, dp, ip]
        L.or_initial_state.argtypes = [vp, dp]
        L.or_rhs.argtypes = [vp, ctypes.c_double, dp, dp]
        L.or_evolve_apply.argtypes = [vp, dp, ctypes.c_double, dp, dp]
        L.or_run.argtypes = [vp, dp, dp, dp, ip]
        L.or_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)] * 1 + [ctypes.POINTER(ctypes.c_longlong)] * 2
        L.or_breaking_log.restype = ctypes.c_char_p
        L.or_breaking_log.argtypes = [vp]
        L.or_reset.argtypes = [vp]
        L.or_fft.argtypes = [ip, dp, dp, dp, dp, ip]
        L.or_mlp_nparams.restype = ip
        L.or_mlp_loss_grad.restype = ctypes.c_double
        L.or_mlp_loss_grad.argtypes = [dp, ctypes.POINTER(ctypes.c_float), ip, dp]
        L.or_jonswap_signal.argtypes = [ctypes.c_double] * 7 + [ctypes.c_ulonglong, dp, ip]
        L.or_kin_dims.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.or_kin_grid.argtypes = [vp, dp, dp]
        L.or_kinematics.argtypes = [vp, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp, dp, dp, dp, dp]
        L.or2d_create.restype = vp
        L.or2d_create.argtypes = [ctypes.POINTER(Or2dTables), ctypes.c_double, ctypes.c_double]
        L.or2d_destroy.argtypes = [vp]
        L.or2d_last_error.restype = ctypes.c_char_p
        L.or2d_rhs.argtypes = [vp, ctypes.c_double, dp, dp]
        L.or2d_evolve_apply.argtypes = [vp, dp, ctypes.c_double, dp, dp]
        L.or2d_run_to.argtypes = [vp, dp, ctypes.c_double, dp, dp]
        L.or2d_stats.argtypes = [vp] + [ctypes.POINTER(ctypes.c_longlong)] * 3
        L.or2d_fft.argtypes = [ip, ip, dp, dp, dp, dp, ip]
        L.or2d_sym.argtypes = [ip, ip, dp, dp]
        L.or2d_set_tprev.argtypes = [vp, ctypes.c_double]
        L.or2d_brk_fields.argtypes = [vp, dp, dp, dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.or2d_brk_log.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ip, ip]
        L.or2d_brk_log_nodes.restype = ctypes.c_longlong
        L.or2d_brk_log_nodes.argtypes = [vp]
        L.or2d_fields.argtypes = [ip, ip, dp, dp, dp, dp]
        L.or2d_run_outputs.argtypes = [vp, dp, dp, dp, ctypes.POINTER(Or2dOutputs)]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    def __init__(self, workdir, eps_abs=0.0, eps_rel=0.0, h0=0.0, t_stop=0.0, seed=0,
                 nref=0, outdir=None, write_fields=0):
        L = lib()
        self._outdir = outdir.encode() if outdir else None
        o = OrOpts(eps_abs, eps_rel, h0, t_stop, seed, nref, write_fields, self._outdir)
        self.h = L.or_create(str(workdir).encode(), ctypes.byref(o))
        if not self.h:
            raise RuntimeError("oracle: " + L.or_last_error().decode())
        self.nx = L.or_nx(self.h)
        self.n = L.or_nt(self.h)

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def scalar(self, name):
        return lib().or_scalar(self.h, name.encode())

    def table(self, name):
        cap = 16 * max(self.nx, self.n) + 16
        out = np.zeros(cap)
        m = lib().or_table(self.h, name.encode(), _p(out), cap)
        if m < 0:
            raise KeyError(name)
        return out[:m].copy()

    def initial_state(self):
        y = np.zeros(4 * self.nx)
        lib().or_initial_state(self.h, _p(y))
        return y

    def kinematics(self, t, tprev, y, dy):
        """kinematic_modul at t for the state y and its RHS dy: dict of eta_cut [nx_out],
        P, dxphi, dzphi, dtdxphi, dtdzphi [nx_out, nz_out], x_out, z_out."""
        L = lib()
        a, b = ctypes.c_int(), ctypes.c_int()
        if L.or_kin_dims(self.h, ctypes.byref(a), ctypes.byref(b)):
            raise RuntimeError("oracle: the deck has no kinematics")
        nxo, nz = a.value, b.value
        xo, zo = np.zeros(nxo), np.zeros(nz)
        L.or_kin_grid(self.h, _p(xo), _p(zo))
        out = {k: np.zeros(nxo * nz) for k in ("P", "dxphi", "dzphi", "dtdxphi", "dtdzphi")}
        ec = np.zeros(nxo)
        y = np.ascontiguousarray(y, dtype=np.float64)
        dy = np.ascontiguousarray(dy, dtype=np.float64)
        if L.or_kinematics(self.h, float(t), float(tprev), _p(y), _p(dy), _p(ec), _p(out["P"]), _p(out["dxphi"]),
                           _p(out["dzphi"]), _p(out["dtdxphi"]), _p(out["dtdzphi"])):
            raise RuntimeError("oracle: " + L.or_last_error().decode())
        res = {k: v.reshape(nxo, nz) for k, v in out.items()}
        res.update(eta_cut=ec, x_out=xo, z_out=zo)
        return res

    def rhs(self, t, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        dz = np.zeros_like(y)
        lib().or_rhs(self.h, float(t), _p(y), _p(dz))
        return dz

    def evolve_apply(self, t, t1, h, y):
        tt = np.array([t], dtype=np.float64)
        hh = np.array([h], dtype=np.float64)
        st = lib().or_evolve_apply(self.h, _p(tt), float(t1), _p(hh), _p(y))
        if st:
            raise RuntimeError("oracle evolve failed")
        return float(tt[0]), float(hh[0])

    def run(self, cap_rows=None):
        cap = cap_rows if cap_rows else self.n
        ng = max(int(self.scalar("ngauge")), 1)
        ge = np.zeros(cap * ng)
        gd = np.zeros(cap * ng)
        tim = np.zeros(cap)
        rows = lib().or_run(self.h, _p(ge), _p(gd), _p(tim), cap)
        return tim[:rows], ge[: rows * ng].reshape(rows, ng), gd[: rows * ng].reshape(rows, ng)

    def stats(self):
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        lib().or_stats(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def breaking_log(self):
        return lib().or_breaking_log(self.h).decode()

    def reset(self):
        lib().or_reset(self.h)


def fft(x, sign=-1):
    x = np.asarray(x, dtype=np.complex128)
    n = x.size
    re = np.ascontiguousarray(x.real)
    im = np.ascontiguousarray(x.imag)
    ro = np.zeros(n)
    io = np.zeros(n)
    lib().or_fft(n, _p(re), _p(im), _p(ro), _p(io), sign)
    return ro + 1j * io


def mlp_loss_grad(params, records):
    """FP64 summed loss and parameter gradient of the learned operator's network."""
    P = np.ascontiguousarray(params, dtype=np.float64)
    R = np.ascontiguousarray(records, dtype=np.float32)
    g = np.zeros(lib().or_mlp_nparams())
    n = R.shape[0]
    L = lib().or_mlp_loss_grad(_p(P), R.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n, _p(g))
    return L, g


def jonswap_components_2d(t, Hs, Tp, gamma, s, depth, rn, ru):
    """or2d_jonswap_components: (a, w, k, theta, phi) of the 2D directional influx."""
    L = lib()
    nh = t.size // 2
    out = [np.zeros(nh) for _ in range(5)]
    t = np.ascontiguousarray(t, dtype=np.float64)
    rn = np.ascontiguousarray(rn, dtype=np.float64)
    ru = np.ascontiguousarray(ru, dtype=np.float64)
    L.or2d_jonswap_components(t.size, _p(t), ctypes.c_double(Hs), ctypes.c_double(Tp), ctypes.c_double(gamma),
                              ctypes.c_double(s), ctypes.c_double(depth), _p(rn), _p(ru), *[_p(o) for o in out])
    return tuple(out)


def directional_signal_2d(t, y, y0, comps, mdir=0.0, ramp_t=None, ramp_y=None):
    """or2d_directional_signal: the direct sum, [lines][nt] elevation and quadrature."""
    L = lib()
    t = np.ascontiguousarray(t, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    a, w, k, th, ph = (np.ascontiguousarray(v, dtype=np.float64) for v in comps)
    rt = np.ones(t.size) if ramp_t is None else np.ascontiguousarray(ramp_t, dtype=np.float64)
    ry = np.ones(y.size) if ramp_y is None else np.ascontiguousarray(ramp_y, dtype=np.float64)
    eta, skew = np.zeros((y.size, t.size)), np.zeros((y.size, t.size))
    L.or2d_directional_signal(t.size, _p(t), y.size, _p(y), ctypes.c_double(y0), a.size, _p(a), _p(w), _p(k),
                              _p(th), _p(ph), ctypes.c_double(mdir), _p(rt), _p(ry), _p(eta), _p(skew))
    return eta, skew


class Oracle2D:
    """The 2D flat-bottom restatement (oracle/hw_oracle2d.c) on a table dict."""

    def __init__(self, tables, eps_abs=0.0, eps_rel=0.0):
        L = lib()
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
        scal = {k: float(tables.get(k, 0.0)) for k in BRK_SCALARS}
        tb = Or2dTables(nx=int(tables["nx"]), ny=int(tables["ny"]), model=int(tables.get("model", 2)),
                        propagation=int(tables.get("propagation", 0)), cpeak=float(tables["cpeak"]),
                        nt=int(tables.get("nt", 0) if keep["sig"] is not None else 0), breaking=brk, **scal,
                        refl_coef=float(tables.get("refl_coef", 0.0)),
                        nrefk=int(tables.get("nrefk", 0)),
                        **{k: (None if v is None else _p(v)) for k, v in keep.items()})
        self.h = L.or2d_create(ctypes.byref(tb), eps_abs, eps_rel)
        if not self.h:
            raise RuntimeError("oracle2d: " + L.or2d_last_error().decode())
        self.nx, self.ny = int(tables["nx"]), int(tables["ny"])
        self.n = self.nx * self.ny

    def close(self):
        if self.h:
            lib().or2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rhs(self, t, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(6 * self.n)
        if lib().or2d_rhs(self.h, float(t), _p(y), _p(out)):
            raise RuntimeError("oracle2d: non-finite RHS")
        return out

    def evolve_apply(self, t, t1, h, y):
        tt, hh = ctypes.c_double(t), ctypes.c_double(h)
        if lib().or2d_evolve_apply(self.h, ctypes.byref(tt), float(t1), ctypes.byref(hh), _p(y)):
            raise RuntimeError("oracle2d: " + lib().or2d_last_error().decode())
        return tt.value, hh.value

    def run_to(self, t, t1, h, y):
        tt, hh = ctypes.c_double(t), ctypes.c_double(h)
        if lib().or2d_run_to(self.h, ctypes.byref(tt), float(t1), ctypes.byref(hh), _p(y)):
            raise RuntimeError("oracle2d: " + lib().or2d_last_error().decode())
        return tt.value, hh.value

    def stats(self):
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        lib().or2d_stats(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return {"rhs_calls": a.value, "accepted": b.value, "rejected": c.value}

    def set_tprev(self, t):
        lib().or2d_set_tprev(self.h, float(t))

    def breaking_fields(self):
        """B, Sb_xhat, Sb_yhat (complex [ny, nx]), flagbr, tracked crests."""
        B = np.zeros(self.n)
        sx, sy = np.zeros(2 * self.n), np.zeros(2 * self.n)
        fl, nc = ctypes.c_int(), ctypes.c_int()
        if lib().or2d_brk_fields(self.h, _p(B), _p(sx), _p(sy), ctypes.byref(fl), ctypes.byref(nc)):
            raise RuntimeError("oracle2d: no breaking")
        shp = (self.ny, self.nx)
        return (B.reshape(shp), (sx[0::2] + 1j * sx[1::2]).reshape(shp), (sy[0::2] + 1j * sy[1::2]).reshape(shp),
                fl.value, nc.value)

    def breaking_log(self):
        """breaking.dat records as a list of (t, [(x, y), ...])."""
        L = lib()
        nn = int(L.or2d_brk_log_nodes(self.h))
        nr = L.or2d_brk_log(self.h, None, None, None, 0, 0)
        t = np.zeros(max(nr, 1))
        cnt = np.zeros(max(nr, 1), dtype=np.int32)
        nodes = np.zeros(2 * max(nn, 1), dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        L.or2d_brk_log(self.h, _p(t), cnt.ctypes.data_as(ip), nodes.ctypes.data_as(ip), nr, nn)
        out, off = [], 0
        for r in range(nr):
            c = int(cnt[r])
            out.append((float(t[r]), [tuple(v) for v in nodes[2 * off:2 * (off + c)].reshape(-1, 2).tolist()]))
            off += c
        return out


class Or2dOutputs(ctypes.Structure):
    """or2d_outputs (oracle/hw_oracle2d.h)."""
    _fields_ = [
        ("outdir", ctypes.c_char_p), ("nt", ctypes.c_int), ("tout", ctypes.POINTER(ctypes.c_double)),
        ("dt", ctypes.c_double), ("npartition", ctypes.c_int), ("uv_every_sample", ctypes.c_int),
        ("hs", ctypes.c_double), ("kp", ctypes.c_double), ("wp", ctypes.c_double),
        ("x", ctypes.POINTER(ctypes.c_double)), ("y", ctypes.POINTER(ctypes.c_double)),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("kx", ctypes.POINTER(ctypes.c_double)), ("ky", ctypes.POINTER(ctypes.c_double)),
        ("bathy", ctypes.POINTER(ctypes.c_double)), ("cfsa", ctypes.POINTER(ctypes.c_double)),
        ("chiadjphi", ctypes.POINTER(ctypes.c_double)),
        ("ngauge", ctypes.c_int), ("xgauge", ctypes.POINTER(ctypes.c_double)),
        ("ygauge", ctypes.POINTER(ctypes.c_double)),
    ]


def run_outputs2d(ora, t, h, z, outdir, tout, dt, npartition, x, y, dx, dy, kx, ky, bathy, cfsa, chiadjphi=None,
                  hs=0.0, kp=0.0, wp=0.0, gauges=None, uv_every_sample=False):
    """or2d_run_outputs on an Oracle2D from (t, h, z); the state z is advanced in
    place.  Returns (samples written, t, h)."""
    keep = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in
            dict(tout=tout, x=x, y=y, kx=kx, ky=ky, bathy=bathy, cfsa=cfsa).items()}
    keep["chiadjphi"] = None if chiadjphi is None else np.ascontiguousarray(chiadjphi, dtype=np.float64)
    g = np.zeros((0, 2)) if gauges is None else np.asarray(gauges, dtype=np.float64).reshape(-1, 2)
    keep["xgauge"], keep["ygauge"] = np.ascontiguousarray(g[:, 0]), np.ascontiguousarray(g[:, 1])
    od = os.path.join(str(outdir), "").encode()
    spec = Or2dOutputs(outdir=od, nt=len(keep["tout"]), dt=float(dt), npartition=int(npartition),
                       uv_every_sample=int(bool(uv_every_sample)), hs=float(hs), kp=float(kp), wp=float(wp),
                       dx=float(dx), dy=float(dy), ngauge=len(g),
                       **{k: (None if keep[k] is None or (k in ("xgauge", "ygauge") and not len(g)) else _p(keep[k]))
                          for k in ("tout", "x", "y", "kx", "ky", "bathy", "cfsa", "chiadjphi", "xgauge", "ygauge")})
    tt, hh = ctypes.c_double(t), ctypes.c_double(h)
    r = lib().or2d_run_outputs(ora.h, ctypes.byref(tt), ctypes.byref(hh), _p(z), ctypes.byref(spec))
    if r < 0:
        raise RuntimeError("oracle2d: " + lib().or2d_last_error().decode())
    return r, tt.value, hh.value


def fields2d(nx, ny, y):
    """eta, u, v ([ny, nx]) of a state: ifftw_2d_c2r of each spectrum."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = [np.zeros(nx * ny) for _ in range(3)]
    lib().or2d_fields(nx, ny, _p(y), *[_p(a) for a in out])
    return tuple(a.reshape(ny, nx) for a in out)


def fft2(x, sign=-1):
    x = np.asarray(x, dtype=np.complex128)
    ny, nx = x.shape
    re = np.ascontiguousarray(x.real).ravel()
    im = np.ascontiguousarray(x.imag).ravel()
    ro, io = np.zeros(nx * ny), np.zeros(nx * ny)
    lib().or2d_fft(nx, ny, _p(re), _p(im), _p(ro), _p(io), sign)
    return (ro + 1j * io).reshape(ny, nx)


def sym2(x):
    x = np.asarray(x, dtype=np.complex128)
    ny, nx = x.shape
    re = np.ascontiguousarray(x.real).ravel().copy()
    im = np.ascontiguousarray(x.imag).ravel().copy()
    lib().or2d_sym(nx, ny, _p(re), _p(im))
    return (re + 1j * im).reshape(ny, nx)


def jonswap_signal(T0, Tend, dt, Tp, Hs, gamma, nTramp, seed):
    """The oracle's seeded jonswap_influx (1d/influx_lib.c:137-255)."""
    L = lib()
    nt = L.or_jonswap_signal(T0, Tend, dt, Tp, Hs, gamma, nTramp, seed, None, 0)
    out = np.zeros(nt)
    L.or_jonswap_signal(T0, Tend, dt, Tp, Hs, gamma, nTramp, seed, _p(out), nt)
    return out

