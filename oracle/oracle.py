"""ctypes wrapper of the FP64 CPU oracle (oracle/hk_oracle.c).

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py import this module, and only as the
checker or as the timed CPU baseline.  The product path (libhkb, hkb) never
imports it.

Each wrapper names the reference file:line of the algorithm it restates; see
oracle/hk_oracle.c for the restatement itself.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "libhkoracle.so")
_lib = None

_d = C.c_double
_i = C.c_int
_i64 = C.c_int64
_p = C.c_void_p


def build() -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.hko_grid_x.restype = _d
        L.hko_grid_x.argtypes = [_d, _d, _i64]
        L.hko_grid_nx.restype = _i
        L.hko_grid_nx.argtypes = [_d, _d, _d]
        L.hko_grid_fill.argtypes = [_d, _d, _i64, _p]
        L.hko_bin_keys.argtypes = [_d, _d, _d, _i64, _i, _p, _p]
        L.hko_partition_interp.restype = _i
        L.hko_partition_interp.argtypes = [_p, _p, _i, _d, _p]
        L.hko_prep_hitran.argtypes = [_i64] + [_p] * 9 + [_i, _p, _p, _p] + [
            _d, _d, _d, _d, _i, _d, _d] + [_p] * 4
        L.hko_prep_exomol.argtypes = [_i64, _p, _p, _p, _p, _d, _d, _d, _d, _d,
                                      _d, _d, _d, _i, _d, _d, _p, _p, _p, _p]
        L.hko_windows.argtypes = [_i64, _p, _p, _p, _p, _d, _d, _i64, _i, _d, _p]
        L.hko_erfcx.restype = _d
        L.hko_erfcx.argtypes = [_d]
        L.hko_voigt916.restype = _d
        L.hko_voigt916.argtypes = [_d, _d]
        L.hko_gh2.restype = _d
        L.hko_gh2.argtypes = [_d, _d]
        L.hko_opacity.argtypes = [_i64, _p, _p, _p, _p, _p, _d, _d, _i64, _i64,
                                  _d, _p, _i, _p]
        L.hko_vjp_sums.argtypes = [_i64, _p, _p, _p, _p, _p, _d, _d, _i64, _p, _p, _i, _i]
        L.hko_vandermonde.argtypes = [_i, _i, _p]
        L.hko_qr.argtypes = [_i, _i, _p, _p, _p]
        L.hko_sort_bins.argtypes = [_i64, _p, _i, _p]
        L.hko_find_cut.argtypes = [_p, _i64, _i, _d, _i, _p]
        L.hko_kdist.argtypes = [_p, _i64, _i, _i, _i, _d, _d, _p, _p, _p, _p,
                                _p, _p]
        L.hko_planck.argtypes = [_d, _d, _p, _p]
        L.hko_windows_p.argtypes = [_i64, _p, _p, _p, _p, _d, _d, _i64, _i, _d, _i, _p]
        L.hko_plinth.argtypes = [_i64, _p, _p, _p, _p, _i, _d, _i, _p]
        L.hko_opacity_p.argtypes = [_i64, _p, _p, _p, _p, _p, _d, _d, _i64, _i64, _d, _i, _p,
                                    _p, _p, _i, _p]
        L.hko_means.argtypes = [_p, _p, _i64, _d, _p]
        L.hko_transmission.argtypes = [_p, _i, _i, _p, _d, _i, _d, _p]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ------------------------------------------------------------------ grid

def grid_nx(numin, numax, dnu) -> int:
    """heliosk.cu:448-455."""
    return int(lib().hko_grid_nx(numin, numax, dnu))


def grid_x(numin, dnu, nx) -> np.ndarray:
    """voigt.h:751-768 setX_kernel (x_i = fma(i, dnu, numin))."""
    x = np.empty(nx, np.float64)
    lib().hko_grid_fill(numin, dnu, nx, _ptr(x))
    return x


def bin_keys(numin, numax, dnu, nx, nbins):
    """voigt.h:779-832 binKey_kernel + binIndex_kernel."""
    key = np.empty(nx, np.int32)
    idx = np.empty(nbins + 2, np.int32)
    lib().hko_bin_keys(numin, numax, dnu, nx, nbins, _ptr(key), _ptr(idx))
    return key, idx


def partition(Tq, q, T) -> float:
    """host.h:9-73 readPartition interpolation; raises on its error cases."""
    Tq = _f64(Tq)
    q = _f64(q)
    out = np.zeros(1)
    ok = lib().hko_partition_interp(_ptr(Tq), _ptr(q), len(Tq), T, _ptr(out))
    if not ok:
        raise ValueError(f"partition function not valid for T={T}")
    return float(out[0])


# ------------------------------------------------------------- line prep

def prep_hitran(lines: dict, iso_mass, iso_ab, iso_Q, T, P, qalphaL=1.0,
                gammaF=1.0, units=0, meanMass=None, Sscale=1.0):
    """host.h:598-649 readFile + voigt.h:331-363 S2_kernel.

    lines: dict of float64 arrays nu, S, EL, A, delta, gair, gself, n and an
    int32 array iso (isotopologue index).  Returns (nu, S, ialphaD, vy).
    """
    n = len(lines["nu"])
    iso_mass = _f64(iso_mass)
    iso_ab = _f64(iso_ab)
    iso_Q = _f64(iso_Q)
    if meanMass is None:
        meanMass = float(np.sum(iso_ab * iso_mass) * Sscale)
    cols = [_f64(lines[k]) for k in ("nu", "S", "EL", "A", "delta", "gair",
                                     "gself", "n")]
    iso = np.ascontiguousarray(lines.get("iso", np.zeros(n, np.int32)),
                               dtype=np.int32)
    outs = [np.empty(n, np.float64) for _ in range(4)]
    lib().hko_prep_hitran(n, *[_ptr(c) for c in cols], _ptr(iso), len(iso_mass),
                          _ptr(iso_mass), _ptr(iso_ab), _ptr(iso_Q), T, P,
                          qalphaL, gammaF, units, meanMass, Sscale,
                          *[_ptr(o) for o in outs])
    return tuple(outs)


def prep_exomol(lines: dict, mass, ab, Q, defaultL, defaultn, T, P,
                gammaF=1.0, units=0, meanMass=None, Sscale=1.0):
    """voigt.h:484-504 L_kernelExomol + voigt.h:365-397 Sf_kernel."""
    n = len(lines["nu"])
    if meanMass is None:
        meanMass = ab * mass * Sscale
    cols = [_f64(lines[k]) for k in ("nu", "S", "EL", "A")]
    outs = [np.empty(n, np.float64) for _ in range(4)]
    lib().hko_prep_exomol(n, *[_ptr(c) for c in cols], mass, ab, Q, defaultL,
                          defaultn, T, P, gammaF, units, meanMass, Sscale,
                          *[_ptr(o) for o in outs])
    return tuple(outs)


def windows(nu, S, iad, vy, numin, dnu, nx, cutMode, cut, profile=1) -> np.ndarray:
    """Per-line index windows (n, 6): i0, b0, c0, c1, b1, i1.

    Restates the region classes of voigt.h:2205-2341 and the per-pair
    predicates of voigt.h:1223, 1481, 1662 as exact FP64 index ranges;
    profiles 2-4 have no regions B and C.
    """
    nu, S, iad, vy = map(_f64, (nu, S, iad, vy))
    n = len(nu)
    win = np.empty((n, 6), np.int64)
    lib().hko_windows_p(n, _ptr(nu), _ptr(S), _ptr(iad), _ptr(vy), numin, dnu,
                        nx, cutMode, cut, int(profile), _ptr(win))
    return win


def plinth(S, iad, vy, win, cutMode, cut, profile=1):
    """Per-line profile value at the cut edge (Plinth_kernel voigt.h:1091-1164)."""
    S, iad, vy = map(_f64, (S, iad, vy))
    win = np.ascontiguousarray(win, dtype=np.int64)
    out = np.empty(len(S), np.float64)
    lib().hko_plinth(len(S), _ptr(S), _ptr(iad), _ptr(vy), _ptr(win), cutMode, cut, int(profile),
                     _ptr(out))
    return out


def erfcx(y: float) -> float:
    return float(lib().hko_erfcx(y))


def voigt916(x: float, y: float) -> float:
    """voigt.h:278-300 voigt_916 (FP64, def_TOL)."""
    return float(lib().hko_voigt916(x, y))


def gh2(x: float, y: float) -> float:
    """voigt.h:1481-1490 region-B rational (t4)."""
    return float(lib().hko_gh2(x, y))


def sublorentz_params(p14, T):
    """{sigma1..3, B1..B3, lo, hi} from the 14 file values (sigma1..3, alpha,
    beta, epsilon of B1..B3, lo, hi) at temperature T (voigt.h:12-35)."""
    p = [float(v) for v in p14]
    B = [p[3 + 3 * k] + p[4 + 3 * k] * np.exp(-p[5 + 3 * k] * T) for k in range(3)]
    return np.array(p[0:3] + B + p[12:14], np.float64)


def opacity(nu, S, iad, vy, win, numin, dnu, nx, kmin=0.0, nthreads=0,
            irange=None, profile=1, plinth=None, sublorentz=None):
    """Line6fA/B/C + AddKStreams restated: K = kmin + sum of contributions.

    irange=(ib, ie) evaluates only grid indices ib <= i < ie of the nx-point
    grid.  Returns (K, pairs) with pairs = (A, B, C) pair counts.
    """
    nu, S, iad, vy = map(_f64, (nu, S, iad, vy))
    win = np.ascontiguousarray(win, dtype=np.int64)
    ib, ie = irange if irange is not None else (0, nx)
    K = np.empty(ie - ib, np.float64)
    pairs = np.zeros(3, np.int64)
    pl = None if plinth is None else _f64(plinth)
    sl = None if sublorentz is None else _f64(sublorentz)
    lib().hko_opacity_p(len(nu), _ptr(nu), _ptr(S), _ptr(iad), _ptr(vy),
                        _ptr(win), numin, dnu, ib, ie, kmin, int(profile), _ptr(pl),
                        _ptr(sl), _ptr(K), nthreads, _ptr(pairs))
    return K, tuple(int(p) for p in pairs)


# ---------------------------------------------------------- k-distribution

def qr(nxb: int, nc: int):
    """resample.h:14-37 Vandermonde + resample.h:73-227 QR_kernel."""
    V = np.empty(nxb * nc, np.float64)
    Cv = np.empty(nc, np.float64)
    D = np.empty(nc, np.float64)
    lib().hko_vandermonde(nxb, nc, _ptr(V))
    lib().hko_qr(nxb, nc, _ptr(V), _ptr(Cv), _ptr(D))
    return V, Cv, D


def sort_bins(K, bin_index, nbins):
    """heliosk.cu:2046-2051 per-bin ascending sort (returns a copy)."""
    K = _f64(K).copy()
    bi = np.ascontiguousarray(bin_index, dtype=np.int32)
    lib().hko_sort_bins(len(K), _ptr(bi), nbins, _ptr(K))
    return K


def kdist(K_sorted, nxb, nbins, nc, kmin=0.0, unitScale=1.0, recon=False,
          qr_mats=None):
    """heliosk.cu:2139-2193 chain (findCut, rescale, lnK, leastSquare[, expfx]).

    Returns (coeff[nbins, nc], nxmin[nbins], recon or None).
    """
    K = _f64(K_sorted).copy()
    nx = len(K)
    V, Cv, D = qr_mats if qr_mats is not None else qr(nxb, nc)
    coeff = np.empty(nbins * nc, np.float64)
    nxmin = np.empty(nbins, np.int32)
    rec = np.empty(nx, np.float64) if recon else None
    lib().hko_kdist(_ptr(K), nx, nxb, nbins, nc, kmin, unitScale, _ptr(V),
                    _ptr(Cv), _ptr(D), _ptr(nxmin), _ptr(coeff), _ptr(rec))
    return coeff.reshape(nbins, nc), nxmin, rec


def planck(nu, T):
    """(B, dB/dT) of resample.h:635-663 at wavenumber nu (cm^-1)."""
    b = np.zeros(1)
    r = np.zeros(1)
    lib().hko_planck(float(nu), float(T), _ptr(b), _ptr(r))
    return float(b[0]), float(r[0])


def means(x, K, T):
    """[sum B K, sum (dB/dT)/K, sum B, sum dB/dT] with the reference's end
    weights (resample.h:635-773); Planck mean = [0]/[2], Rosseland = [3]/[1]."""
    x = _f64(x)
    K = _f64(K)
    out = np.zeros(4)
    lib().hko_means(_ptr(x), _ptr(K), len(K), float(T), _ptr(out))
    return out


def transmission(K, nxb, nbins, nxmin=None, kmin=0.0, nTr=1000, dTr=0.05):
    """Tr[nbins, nTr] of resample.h:541-608 from per-bin K (sorted or
    reconstructed); m_j = exp((j - nTr // 2) dTr)."""
    K = _f64(K)
    nm = None if nxmin is None else np.ascontiguousarray(nxmin, dtype=np.int32)
    Tr = np.empty(nbins * nTr)
    lib().hko_transmission(_ptr(K), nxb, nbins, _ptr(nm), float(kmin), nTr, float(dTr), _ptr(Tr))
    return Tr.reshape(nbins, nTr)


def state_opacity(lines, iso_mass, iso_ab, iso_Q, T, P, numin, numax, dnu,
                  cutMode=0, cut=25.0, kmin=0.0, qalphaL=1.0, gammaF=1.0,
                  nthreads=0):
    """Whole forward path for one HITRAN-format state: prep, windows, sum."""
    nx = grid_nx(numin, numax, dnu)
    nu, S, iad, vy = prep_hitran(lines, iso_mass, iso_ab, iso_Q, T, P,
                                 qalphaL=qalphaL, gammaF=gammaF)
    win = windows(nu, S, iad, vy, numin, dnu, nx, cutMode, cut)
    K, pairs = opacity(nu, S, iad, vy, win, numin, dnu, nx, kmin, nthreads)
    return K, pairs, (nu, S, iad, vy, win)


# ------------------------------------------------------ reference gradient

_H, _C, _KB, _T0 = 6.62606957e-27, 2.99792458e10, 1.3806489e-16, 296.0


def vjp_sums(nu, S, iad, vy, win, numin, dnu, nx, u, nthreads=0, profile=1):
    """hko_vjp_sums: (4, n) per-line sums of the vector-Jacobian product of
    K (G_S, G_y, G_x, G_n), FP64.  Profiles 3-4 have no y dependence
    (G_y = 0) and their G_x includes the dependence on iad through the grid
    step vb = dnu iad (binned Gaussian)."""
    n = len(nu)
    nu, S, iad, vy, u = map(_f64, (nu, S, iad, vy, u))
    win = np.ascontiguousarray(win, dtype=np.int64)
    G = np.zeros(4 * n, np.float64)
    lib().hko_vjp_sums(n, _ptr(nu), _ptr(S), _ptr(iad), _ptr(vy), _ptr(win), numin, dnu, nx,
                       _ptr(u), _ptr(G), int(profile), nthreads)
    return G.reshape(4, n)


def partition_dlnq(Tq, q, T):
    """d ln Q / dT of the linear interpolant of host.h:9-73: the slope of the
    segment holding T (the mean of the two slopes at a table node) over Q."""
    Tq, q = _f64(Tq), _f64(q)
    Q = partition(Tq, q, T)
    j = int(np.searchsorted(Tq, T, side="left"))
    j = min(max(j, 1), len(Tq) - 1)
    slope = (q[j] - q[j - 1]) / (Tq[j] - Tq[j - 1])
    if T == Tq[j] and j + 1 < len(Tq):
        slope = 0.5 * (slope + (q[j + 1] - q[j]) / (Tq[j + 1] - Tq[j]))
    return slope / Q


def vjp_hitran(lines, mass, Tq, Qq, T, P, u, numin, dnu, nx, cut=25.0, qalphaL=1.0,
               s_scale=None, g_scale=None, profile=1, cutMode=0):
    """FP64 reference gradient of a loss with seed u = dLoss/dK (one HITRAN
    isotopologue; the windows of cutMode at the state, held fixed: a window
    edge that moves with T or P is not differentiated): returns (dT, dP, dlogS per line, dgammaL per
    line), by the chain rule of the line scaling of prep_hitran applied to
    the per-line sums of vjp_sums.  Optional per-line multipliers of the
    strength and of the Lorentz width, as the library's hk_set_line_scales.
    profiles 2-4: windows without regions B and C; every point takes the
    profile's region-A term (Lorentz, Doppler, binned Gaussian)."""
    Q = partition(Tq, Qq, T)
    nu, S, iad, vy = prep_hitran(lines, [mass], [1.0], [Q], T, P, qalphaL=qalphaL)
    if s_scale is not None:
        S = S * s_scale
    if g_scale is not None:
        vy = vy * g_scale
    win = windows(nu, S, iad, vy, numin, dnu, nx, cutMode, cut, profile=profile)
    gS, gy, gx, gn = vjp_sums(nu, S, iad, vy, win, numin, dnu, nx, u, profile=profile)
    c = _H * _C / _KB
    el = _f64(lines["EL"])
    delta = _f64(lines["delta"])
    ne = _f64(lines["n"])
    At = _f64(lines["A"]) / (4.0 * np.pi * _C)
    gs = np.ones_like(nu) if g_scale is None else _f64(g_scale)
    dlnQ = partition_dlnq(Tq, Qq, T)
    e1, e0 = np.exp(-c * nu / T), np.exp(-c * nu / _T0)
    dlS_dT = -dlnQ + c * el / T**2 - (c * nu / T**2) * e1 / (1 - e1) - 0.5 / T
    dlS_dnu = (c / T) * e1 / (1 - e1) - (c / _T0) * e0 / (1 - e0) - 1.0 / nu
    gam = (1.0 - qalphaL) * _f64(lines["gair"]) + qalphaL * _f64(lines["gself"])
    pb = (_T0 / T) ** ne
    aLc = gs * gam * P * pb
    aL = gs * (gam * P * pb + At)
    daL_dT = -ne * aLc / T
    daL_dP = gs * gam * pb
    diad_dT = -0.5 * iad / T
    diad_dP = -iad * delta / nu
    dy_dT = daL_dT * iad + aL * diad_dT
    dy_dP = daL_dP * iad + aL * diad_dP
    ok = (S != 0) & (iad > 0)
    gI = np.where(ok, gx / np.where(ok, iad, 1.0), 0.0)
    gN = -gn * iad
    dT = float(np.sum(np.where(ok, gS * dlS_dT + gy * dy_dT + gI * diad_dT, 0.0)))
    dP = float(np.sum(np.where(ok, gS * dlS_dnu * delta + gy * dy_dP + gI * diad_dP + gN * delta, 0.0)))
    return dT, dP, gS, gy * iad


# ------------------------------------------------------------------ CIA
AMAGAT = 2.6867774e19  # define.h:43
NA = 6.0221412927e23


def cia_opacity(path, nsets, mass1, x, T, P, kmin=0.0):
    """readCiaFile (host.h:670-785) restated as it reads the file: per set a
    fixed-width header (20, 10, 10, 7, 7, 10 characters, then 36 skipped),
    linear interpolation in nu inside [nu0, nu1), the last set with
    T_set <= T taken as is and the first set above T interpolated linearly
    in T from the value left by the sets before; stop after that set; K =
    cia * rho (P 273.15 / T amagat) * NA / mass1 + kmin, or kmin everywhere
    when T is above the last set read.  x: the grid (FP64 array)."""
    x = np.asarray(x, np.float64)
    K = np.zeros(len(x))
    with open(path, "r") as f:
        data = f.read()
    pos = 0

    def fgets(n):  # C fgets(buf, n): up to n-1 characters, stops after a newline
        nonlocal pos
        end = data.find("\n", pos, pos + n - 1)
        end = pos + n - 1 if end < 0 else end + 1
        out = data[pos:end]
        pos = end
        return out

    def scan_double():
        nonlocal pos
        while pos < len(data) and data[pos].isspace():
            pos += 1
        start = pos
        while pos < len(data) and not data[pos].isspace():
            pos += 1
        return float(data[start:pos])

    Tcia1 = 0.0
    for _ in range(nsets):
        Tcia0 = Tcia1
        fgets(21)
        fgets(11)
        c2 = fgets(11)
        c3 = fgets(8)
        c4 = fgets(8)
        fgets(11)
        fgets(37)
        ncia = int(c3)
        Tcia1 = float(c4)
        numax = float(c2)
        nu0 = scan_double()
        cia0 = scan_double()
        nu1 = scan_double()
        cia1 = scan_double()
        nc = 2
        for i in range(len(x)):
            while x[i] >= nu1:
                nu0, cia0 = nu1, cia1
                nu1 = scan_double()
                cia1 = scan_double()
                nc += 1
                if nc == ncia:
                    break
            if nu0 <= x[i] < nu1:
                if Tcia1 <= T:
                    K[i] = cia0 + (cia1 - cia0) * (x[i] - nu0) / (nu1 - nu0)
                if T < Tcia1 and Tcia0 > 0.0:
                    K0 = K[i]
                    K1 = cia0 + (cia1 - cia0) * (x[i] - nu0) / (nu1 - nu0)
                    K[i] = K0 + (K1 - K0) * (T - Tcia0) / (Tcia1 - Tcia0)
            if nu1 == numax:
                break
            if i == len(x) - 1:
                while nc < ncia:
                    nu1 = scan_double()
                    cia1 = scan_double()
                    nc += 1
        fgets(3)
        if T <= Tcia1:
            break
    rho1 = P * 273.15 / T * AMAGAT
    if Tcia1 < T:
        return np.full(len(x), kmin)
    K = K * rho1
    K = K * (NA / mass1)  # host.h:779: K *= def_NA / cia.mass1
    return K + kmin
