"""hkb -- Python binding of libhkb, the B200 (sm_100a) HELIOS-K opacity engine.

A thin ctypes layer over the C ABI in include/hkb.h.  Host arrays are numpy;
device buffers are torch CUDA tensors (plumbing only: torch supplies device
memory and streams, every computation runs in libhkb's own kernels).

There is no CPU fallback: importing works anywhere, but creating a Context
needs a CUDA device and the built library (helios-k_b200/lib/libhkb.so);
both missing conditions raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
# HKB_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("HKB_LIB", os.path.join(os.path.dirname(_PKG), "lib", "libhkb.so"))
HEADER_PATH = os.path.join(os.path.dirname(os.path.dirname(_PKG)), "include", "hkb.h")

HK_OK = 0
STATUS_NAMES = {0: "HK_OK", -1: "HK_ERR_ARG", -2: "HK_ERR_IO", -3: "HK_ERR_FORMAT",
                -4: "HK_ERR_RANGE", -5: "HK_ERR_CUDA", -6: "HK_ERR_STATE",
                -7: "HK_ERR_NOMEM", -8: "HK_ERR_UNSUPPORTED", -9: "HK_ERR_TIMEOUT"}
PLAIN_FP64 = 0
MIXED = 1
HITRAN = 0
EXOMOL = 2

_lib = None
_p = C.c_void_p
_d = C.c_double
_i = C.c_int
_i64 = C.c_int64


class HkError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib():
    """Load libhkb.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libhkb.so not built: {LIB_PATH} (run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        sig = {
            "hk_create": (_p, [_i, C.POINTER(_i)]),
            "hk_destroy": (None, [_p]),
            "hk_last_error": (C.c_char_p, [_p]),
            "hk_version": (C.c_char_p, []),
            "hk_set_species": (_i, [_p, _i, _i, _p, _p, _d, _d]),
            "hk_set_partition": (_i, [_p, _i, _i, _p, _p]),
            "hk_set_options": (_i, [_p, _d, _d, _i, _d]),
            "hk_load_lines_hitran": (_i, [_p, _i64] + [_p] * 9),
            "hk_load_lines_exomol": (_i, [_p, _i64] + [_p] * 4),
            "hk_load_species_file": (_i, [_p, C.c_char_p, C.c_char_p, _d, _d, _i, _d]),
            "hk_num_lines": (_i64, [_p]),
            "hk_set_grid": (_i, [_p, _d, _d, _d, _i, _i, _d, _d]),
            "hk_grid_points": (_i64, [_p]),
            "hk_opacity": (_i, [_p, _i, _p, _p, _i, _p, _i, _p]),
            "hk_kdist": (_i, [_p, _i, _p, _i, _i, _d, _p, _p, _p, _p, _i, _p]),
            "hk_state_lines": (_i, [_p, _d, _d, _p, _p, _p, _p, _p]),
            "hk_line_order": (_i, [_p, _p]),
            "hk_profile_eval": (_i, [_p, _i64, _p, _p, _i, _p]),
            "hk_last_timing": (_i, [_p, _p, _p]),
            "hk_tile_points": (_i, []),
            "hk_fp32_peak": (_i, [_p, _p]),
            "hk_kdist_noalloc": (_i, [_p, _i, _i64, _i, _i, _d, _d, _p, _p, _p, _p,
                                      C.c_char_p, _i]),
            "hk_set_line_scales": (_i, [_p, _p, _p]),
            "hk_set_line_scales_device": (_i, [_p, _p, _p, _p]),
            "hk_set_workspace": (_i, [_p, _d, _d]),
            "hk_opacity_vjp": (_i, [_p, _d, _d, _i, _p, _i, _p, _p, _p, _p, _i, _p]),
            "hk_opacity_vjp_log": (_i, [_p, _d, _d, _i, _p, _i, _p, _p, _p, _p, _i, _p]),
            "hk_table_build": (_i, [_p, _i, _p, _p, _i, _p, _i, _d, _p, _p]),
            "hk_table_run": (_i, [_p, _p]),
            "hk_table_status": (_i, [_p, _p]),
            "hk_set_table_mode": (_i, [_p, _i]),
            "hk_table_free": (_i, [_p]),
            "hk_table_kernels": (_i64, [_p]),
            "hk_last_launches": (_i64, [_p]),
            "hk_count_pairs": (_i, [_p, _d, _d, _p]),
            "hk_num_tile_shapes": (_i, []),
            "hk_tile_shape_info": (_i, [_i, _p, _p, _p]),
            "hk_set_tuning": (_i, [_p, _i]),
            "hk_set_tile_shape": (_i, [_p, _i]),
            "hk_tuning_result": (_i, [_p, _p, _p, _p]),
            "hk_means": (_i, [_p, _i, _p, _p, _i, _p, _i, _p]),
            "hk_set_profile": (_i, [_p, _i, _i]),
            "hk_set_sublorentzian": (_i, [_p, _p]),
            "hk_load_mixture": (_i, [_p, C.c_char_p, _i, _p, _p, _d, _d, _i, _d]),
            "hk_load_cia": (_i, [_p, C.c_char_p, C.c_char_p, _p]),
            "hk_transmission": (_i, [_p, _i, _p, _p, _i, _i, _d, _p, _i, _p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def header_functions(path: str = HEADER_PATH):
    """Names of the functions declared in include/hkb.h."""
    import re
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hk_[a-z_0-9]+)\s*\(", txt)))


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _is_dev(t):
    return hasattr(t, "is_cuda") and t.is_cuda


def _host_f64(n):
    """A numpy float64 array of n values in page-locked memory when torch
    can supply it (its caching host allocator reuses the block once the
    array is dropped), so a device-to-host copy into it runs at full link
    speed; plain numpy memory otherwise, and above 1 GiB (the allocator
    rounds blocks up to powers of two)."""
    try:
        import torch
        if 8 * n <= (1 << 30) and torch.cuda.is_available():
            return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    except ImportError:
        pass
    return np.empty(n, np.float64)


class Context:
    """One libhkb context bound to one GPU (hk_create / hk_destroy)."""

    def __init__(self, device: int = 0):
        st = C.c_int(0)
        self._h = lib().hk_create(device, C.byref(st))
        if not self._h:
            raise HkError(st.value, f"hk_create(device={device}) failed (no CUDA device?)")
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib().hk_destroy(self._h)
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

    def _chk(self, st):
        if st != HK_OK:
            raise HkError(st, lib().hk_last_error(self._h).decode())

    # ---------------------------------------------------------- setup
    def set_species(self, database, mass, abundance, defaultL=0.0, defaultn=0.0):
        m = _f64(np.atleast_1d(mass))
        a = _f64(np.atleast_1d(abundance))
        self._chk(lib().hk_set_species(self._h, database, len(m), _ptr(m), _ptr(a),
                                       defaultL, defaultn))

    def set_partition(self, iso, T, Q):
        T = _f64(T)
        Q = _f64(Q)
        self._chk(lib().hk_set_partition(self._h, iso, len(T), _ptr(T), _ptr(Q)))

    def set_options(self, qalphaL=0.5, gammaF=1.0, units=0, Sscale=1.0):
        self._chk(lib().hk_set_options(self._h, qalphaL, gammaF, units, Sscale))

    def load_lines_hitran(self, lines: dict):
        n = len(lines["nu"])
        cols = [_f64(lines[k]) for k in ("nu", "S", "EL", "A", "delta", "gair", "gself", "n")]
        iso = lines.get("iso")
        iso = None if iso is None else np.ascontiguousarray(iso, dtype=np.int32)
        self._chk(lib().hk_load_lines_hitran(self._h, n, *[_ptr(c) for c in cols], _ptr(iso)))

    def load_lines_exomol(self, lines: dict):
        n = len(lines["nu"])
        cols = [_f64(lines[k]) for k in ("nu", "S", "EL", "A")]
        self._chk(lib().hk_load_lines_exomol(self._h, n, *[_ptr(c) for c in cols]))

    def load_species_file(self, path, species, numin, numax, cutMode, cut):
        self._chk(lib().hk_load_species_file(self._h, path.encode(), species.encode(),
                                             numin, numax, cutMode, cut))

    def load_mixture(self, path, species, abundances, numin, numax, cutMode, cut):
        """Several species' line files as one line list (SpeciesFile)."""
        names = (C.c_char_p * len(species))(*[x.encode() for x in species])
        ab = _f64(abundances)
        self._chk(lib().hk_load_mixture(self._h, path.encode(), len(species),
                                        C.cast(names, C.c_void_p), _ptr(ab), numin, numax,
                                        cutMode, cut))

    def load_cia(self, path, system):
        """A HITRAN CIA table (<path><system>_2011.cia) in place of lines;
        returns the collider mass of the units = 1 scaling."""
        m = C.c_double(0.0)
        self._chk(lib().hk_load_cia(self._h, path.encode(), system.encode(), C.byref(m)))
        return m.value

    @property
    def num_lines(self):
        return int(lib().hk_num_lines(self._h))

    def set_grid(self, numin, numax, dnu, nbins, cutMode=0, cut=25.0, kmin=0.0):
        self._chk(lib().hk_set_grid(self._h, numin, numax, dnu, nbins, cutMode, cut, kmin))
        self._nbins = nbins

    @property
    def nx(self):
        return int(lib().hk_grid_points(self._h))

    # -------------------------------------------------------- compute
    def opacity(self, T, P, precision=MIXED, out=None, stream=None):
        """K for every state (T[s], P[s]): array (nstates, Nx), FP64.

        out: optional numpy array or torch CUDA tensor (nstates * Nx float64).
        With a CUDA tensor the call is asynchronous on `stream` (a torch
        stream or raw handle; default: torch's current stream).
        """
        T = _f64(np.atleast_1d(T))
        P = _f64(np.atleast_1d(P))
        ns = len(T)
        if out is None:
            out = np.empty((ns, self.nx), np.float64)
        dev = _is_dev(out)
        sh = _stream_handle(stream, dev)
        self._chk(lib().hk_opacity(self._h, ns, _ptr(T), _ptr(P), precision, _ptr(out),
                                   int(dev), sh))
        return out

    def kdist(self, K, nC=20, unitScale=1.0, coeff=True, nxmin=True, sorted_K=False,
              recon=False, stream=None, outputs_on_device=None):
        """Per-bin sort + Chebyshev fit of K (nstates, Nx).

        Returns dict with 'coeff' (nstates, nbins, nC), 'nxmin' (nstates, nbins)
        and optionally 'sorted' / 'recon' (nstates, Nx).
        """
        dev_in = _is_dev(K)
        if not dev_in:
            K = _f64(K)
        ns = K.shape[0] if K.ndim == 2 else 1
        nx = self.nx
        nb = self._nbins
        if outputs_on_device is None:
            outputs_on_device = dev_in
        if outputs_on_device:
            import torch
            mk = lambda shape, dt: torch.empty(shape, dtype=dt, device=K.device)
            f64, i32 = torch.float64, torch.int32
        else:
            mk = lambda shape, dt: np.empty(shape, dt)
            f64, i32 = np.float64, np.int32
        res = {}
        res["coeff"] = mk((ns, nb, nC), f64) if coeff else None
        res["nxmin"] = mk((ns, nb), i32) if nxmin else None
        res["sorted"] = mk((ns, nx), f64) if sorted_K else None
        res["recon"] = mk((ns, nx), f64) if recon else None
        sh = _stream_handle(stream, dev_in or outputs_on_device)
        self._chk(lib().hk_kdist(self._h, ns, _ptr(K), int(dev_in), nC, unitScale,
                                 _ptr(res["coeff"]), _ptr(res["nxmin"]), _ptr(res["sorted"]),
                                 _ptr(res["recon"]), int(outputs_on_device), sh))
        return res

    def set_profile(self, profile=1, remove_plinth=0):
        """1 Voigt, 2 Lorentz, 3 Doppler, 4 binned Gaussian; remove_plinth 1
        subtracts each line's value at its cut edge (FP64 form for 2-4 and
        plinth removal)."""
        self._chk(lib().hk_set_profile(self._h, int(profile), int(remove_plinth)))

    def set_sublorentzian(self, params=None):
        """14 values (sigma1..3, alpha/beta/epsilon of B1..B3, x_lo, x_hi) or
        None to turn the sub-Lorentzian chi factor off."""
        p = None if params is None else _f64(params)
        if p is not None and len(p) != 14:
            raise ValueError("need 14 sub-Lorentzian parameters")
        self._chk(lib().hk_set_sublorentzian(self._h, _ptr(p)))

    # ------------------------------------ mean opacities, transmission
    def means(self, T, K, stream=None):
        """(nstates, 4) sums [B K, (dB/dT)/K, B, dB/dT] over the grid with the
        reference's end weights; Planck mean = [:, 0] / [:, 2], Rosseland
        mean = [:, 3] / [:, 1].  K: (nstates, Nx) numpy or CUDA tensor."""
        T = _f64(np.atleast_1d(T))
        dev = _is_dev(K)
        if not dev:
            K = _f64(K)
        ns = len(T)
        out = np.empty((ns, 4), np.float64)
        sh = _stream_handle(stream, dev)
        self._chk(lib().hk_means(self._h, ns, _ptr(T), _ptr(K), int(dev), _ptr(out), 0, sh))
        return out

    def transmission(self, K, nxmin=None, nTr=1000, dTr=0.05, stream=None):
        """(nstates, nbins, nTr) transmission function of per-bin K (sorted,
        or reconstructed by the fit, with its nxmin)."""
        dev = _is_dev(K)
        if not dev:
            K = _f64(K)
            if nxmin is not None:
                nxmin = np.ascontiguousarray(nxmin, dtype=np.int32)
        ns = K.shape[0] if K.ndim == 2 else 1
        out = np.empty((ns, self._nbins, nTr), np.float64)
        sh = _stream_handle(stream, dev)
        self._chk(lib().hk_transmission(self._h, ns, _ptr(K), _ptr(nxmin), int(dev), int(nTr),
                                        float(dTr), _ptr(out), 0, sh))
        return out

    # ----------------------------------------------------- tile shapes
    def set_tuning(self, mode):
        """0: fixed tile shape; 1: tune when it pays (tables, batches);
        2: tune on the first mixed call of a workload."""
        self._chk(lib().hk_set_tuning(self._h, int(mode)))

    def set_tile_shape(self, shape):
        self._chk(lib().hk_set_tile_shape(self._h, int(shape)))

    def tuning_result(self):
        """(shape of the last mixed call, tuned shape or -1, probe ms per shape)."""
        a = np.zeros(1, np.int32)
        b = np.zeros(1, np.int32)
        ms = np.zeros(num_tile_shapes(), np.float64)
        self._chk(lib().hk_tuning_result(self._h, _ptr(a), _ptr(b), _ptr(ms)))
        return int(a[0]), int(b[0]), ms

    def set_workspace(self, prep_bytes=24 * 2**30, part_bytes=4 * 2**30):
        """Workspace budgets; states above the first run in grid sections."""
        self._chk(lib().hk_set_workspace(self._h, float(prep_bytes), float(part_bytes)))

    # --------------------------------------------------------- adjoint
    def set_line_scales(self, s_scale=None, g_scale=None, stream=None):
        """Per-line multipliers of strength and Lorentz width (load order).

        CUDA tensors (float64 on this context's GPU, or convertible to it)
        are reordered and checked on the GPU, in order on `stream` (default:
        torch's current stream), without passing through host memory
        (hk_set_line_scales_device); anything else goes through the host
        (hk_set_line_scales)."""
        if _is_dev(s_scale) or _is_dev(g_scale):
            import torch
            dev = torch.device("cuda", self.device)
            conv = lambda v: None if v is None else torch.as_tensor(v, dtype=torch.float64, device=dev).contiguous()
            s, g = conv(s_scale), conv(g_scale)
            self._chk(lib().hk_set_line_scales_device(self._h, _ptr(s), _ptr(g),
                                                      _stream_handle(stream, True)))
            return
        s = None if s_scale is None else _f64(s_scale)
        g = None if g_scale is None else _f64(g_scale)
        self._chk(lib().hk_set_line_scales(self._h, _ptr(s), _ptr(g)))

    def opacity_vjp(self, T, P, u, precision=MIXED, per_line=True, stream=None, log_gamma=False,
                    device_out=False):
        """dLoss/dT, dLoss/dP and (per_line) dLoss/dlog S, dLoss/dgammaL for
        the seed u = dLoss/dK (Nx values; numpy or CUDA tensor).  log_gamma:
        the width gradient per log gammaL instead (hk_opacity_vjp_log);
        device_out: the per-line results as CUDA tensors (no host copy)."""
        dev = _is_dev(u)
        if not dev:
            u = _f64(u)
        n = self.num_lines
        dT, dP = C.c_double(0), C.c_double(0)
        if device_out:
            import torch
            mk = lambda: torch.empty(n, dtype=torch.float64, device=torch.device("cuda", self.device))
        else:
            mk = lambda: _host_f64(n)
        dS = mk() if per_line else None
        dG = mk() if per_line else None
        sh = _stream_handle(stream, dev or device_out)
        fn = lib().hk_opacity_vjp_log if log_gamma else lib().hk_opacity_vjp
        self._chk(fn(self._h, float(T), float(P), precision, _ptr(u), int(dev), C.byref(dT),
                     C.byref(dP), _ptr(dS), _ptr(dG), int(device_out), sh))
        return dT.value, dP.value, dS, dG

    # ---------------------------------------------------------- tables
    def table_build(self, T, P, K, coeff, nxmin, nC=20, unitScale=1.0, precision=MIXED):
        """Record the T-P table (states T[s], P[s]) as one CUDA graph.

        K (nstates, Nx) float64, coeff (nstates, nbins, nC) float64 and nxmin
        (nstates, nbins) int32 are torch CUDA tensors that must outlive the
        table."""
        T = _f64(np.atleast_1d(T))
        P = _f64(np.atleast_1d(P))
        for t in (K, coeff, nxmin):
            if not _is_dev(t):
                raise ValueError("table buffers must be CUDA tensors")
        self._table_bufs = (K, coeff, nxmin)
        self._chk(lib().hk_table_build(self._h, len(T), _ptr(T), _ptr(P), precision, _ptr(K),
                                       nC, unitScale, _ptr(coeff), _ptr(nxmin)))

    def set_table_mode(self, fused):
        """0: per-batch launches (default); 1: one persistent launch for the
        line prep and Voigt sums of every state (tables of >= 4 states)."""
        self._chk(lib().hk_set_table_mode(self._h, int(fused)))

    def table_run(self, stream=None):
        """Replay the recorded table (one graph launch, asynchronous)."""
        self._chk(lib().hk_table_run(self._h, _stream_handle(stream, True)))

    def table_status(self, stream=None):
        """Synchronise the stream; raises HkError (status -9) if a bounded
        wait inside the last table run ran out (its results incomplete)."""
        self._chk(lib().hk_table_status(self._h, _stream_handle(stream, True)))

    def table_free(self):
        self._chk(lib().hk_table_free(self._h))
        self._table_bufs = None

    @property
    def table_kernels(self):
        return int(lib().hk_table_kernels(self._h))

    def count_pairs(self, T, P):
        """(A, B, C) pairs of one state inside the cutoff windows."""
        out = np.zeros(3, np.int64)
        self._chk(lib().hk_count_pairs(self._h, float(T), float(P), _ptr(out)))
        return tuple(int(v) for v in out)

    @property
    def last_launches(self):
        return int(lib().hk_last_launches(self._h))

    # ---------------------------------------------------- diagnostics
    def state_lines(self, T, P):
        n = self.num_lines
        outs = [np.empty(n, np.float64) for _ in range(4)]
        win = np.empty((n, 6), np.int64)
        self._chk(lib().hk_state_lines(self._h, T, P, *[_ptr(o) for o in outs], _ptr(win)))
        return (*outs, win)

    def line_order(self):
        o = np.empty(self.num_lines, np.int64)
        self._chk(lib().hk_line_order(self._h, _ptr(o)))
        return o

    def profile_eval(self, x, y, precision=MIXED):
        x = _f64(x)
        y = _f64(y)
        out = np.empty(len(x), np.float64)
        self._chk(lib().hk_profile_eval(self._h, len(x), _ptr(x), _ptr(y), precision, _ptr(out)))
        return out

    def last_timing(self):
        a = C.c_double(-1)
        b = C.c_double(-1)
        self._chk(lib().hk_last_timing(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def fp32_peak_tflops(self):
        t = C.c_double(0)
        self._chk(lib().hk_fp32_peak(self._h, C.byref(t)))
        return t.value


def _stream_handle(stream, device_io):
    if stream is None:
        if not device_io:
            return None
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))


def tile_points() -> int:
    """Grid points per tile of the default shape."""
    return int(lib().hk_tile_points())


def num_tile_shapes() -> int:
    return int(lib().hk_num_tile_shapes())


def tile_shape(shape, warps=False):
    """(lines per staged chunk, grid points per tile[, warps per CTA]) of a
    tile shape."""
    a = np.zeros(1, np.int32)
    b = np.zeros(1, np.int32)
    w = np.zeros(1, np.int32)
    st = lib().hk_tile_shape_info(int(shape), _ptr(a), _ptr(b), _ptr(w))
    if st != HK_OK:
        raise HkError(st, "tile shape %d out of range" % shape)
    return (int(a[0]), int(b[0]), int(w[0])) if warps else (int(a[0]), int(b[0]))

