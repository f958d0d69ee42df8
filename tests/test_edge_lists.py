"""GPU: edge cases of the line list against the FP64 oracle.

* no line reaches the grid (all centres beyond the grid by more than the
  cut): K is exactly 0 in both forms and the fit marks every bin empty;
* single lines at special places: a centre exactly on a grid point (x = 0
  in the region-C evaluators), a line with no Lorentz width (y = 0: the
  Voigt profile is the Gaussian), centres just outside either end of the
  grid whose wings reach into it, and centres exactly on numin and numax.
  Each is run alone (one line, one warp's worth of work in a tile) and all
  together; windows bit-exact, K within 1e-12 (plain FP64) and 1e-5 (mixed)
  relative where K > 1e-6 of its bin maximum, as the parity tests.
The grid step is 2^-7 cm^-1 so that grid points and centres coincide
exactly.
"""
import numpy as np
import pytest

import hkb
import oracle
from hkb import synth
from test_gpu_parity import masked_relerr

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS, CUT = 100.0, 400.0, 2.0 ** -7, 30, 25.0
T, P = 900.0, 0.5


def _lines(nu, gamma=0.05):
    n = len(nu)
    L = synth.hitran_lines(n, seed=2, nu_max=1.0)
    L["nu"] = np.asarray(nu, np.float64)
    L["S"] = np.full(n, 1e-20) * L["S"] / L["S"]
    L["gair"] = np.full(n, gamma)
    L["gself"] = np.full(n, gamma)
    L["EL"] = np.full(n, 500.0)
    return L


def _ctx(L):
    Tq, Qq = synth.q_table()
    ctx = hkb.Context(0)
    ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
    ctx.set_partition(0, Tq, Qq)
    ctx.set_options(qalphaL=1.0)
    ctx.load_lines_hitran(L)
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, CUT)
    return ctx


def _oracle(L):
    Tq, Qq = synth.q_table()
    Q = oracle.partition(Tq, Qq, T)
    nu, S, iad, vy = oracle.prep_hitran(L, [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, CUT)
    K, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx)
    return K, win


def test_no_line_reaches_the_grid():
    L = _lines([10.0, 50.0, NUMIN - CUT - 1.0, NUMAX + CUT + 1.0, 900.0])
    with _ctx(L) as ctx:
        nx = ctx.nx
        for prec in (hkb.MIXED, hkb.PLAIN_FP64):
            K = ctx.opacity([T], [P], prec)
            assert K.shape == (1, nx) and np.all(K == 0.0)
        r = ctx.kdist(K, nC=20)
        Kref, _ = _oracle(L)
        assert np.all(Kref == 0.0)
        key, idx = oracle.bin_keys(NUMIN, NUMAX, DNU, nx, NBINS)
        co, nxmin, _ = oracle.kdist(oracle.sort_bins(Kref, idx, NBINS), nx // NBINS, NBINS, 20)
        assert np.array_equal(r["nxmin"][0], nxmin)
        assert np.all(nxmin == nx // NBINS)


SPECIAL = {
    "on_grid_point": ([250.0], 0.0005),  # y ~ 0.3: region C holds x = 0
    "no_lorentz_width": ([250.0 + 0.3 * DNU], 0.0),
    "left_of_grid": ([NUMIN - 3.0], 0.05),
    "right_of_grid": ([NUMAX + 3.0], 0.05),
    "on_numin": ([NUMIN], 0.05),
    "on_numax": ([NUMAX], 0.05),
}


@pytest.mark.parametrize("case", list(SPECIAL) + ["all"])
def test_single_lines_at_special_places(case):
    if case == "all":
        nu = [v[0][0] for v in SPECIAL.values()]
        L = _lines(nu)
        for j, (_, gamma) in enumerate(SPECIAL.values()):
            L["gair"][j] = L["gself"][j] = gamma
    else:
        nu, gamma = SPECIAL[case]
        L = _lines(nu, gamma)
    Kref, win = _oracle(L)
    with _ctx(L) as ctx:
        gnu, gS, giad, gvy, gwin = ctx.state_lines(T, P)
        order = ctx.line_order()
        assert np.array_equal(gwin, win[order])
        assert np.any(Kref > 0.0)
        for prec, tol in ((hkb.PLAIN_FP64, 1e-12), (hkb.MIXED, 1e-5)):
            K = ctx.opacity([T], [P], prec)[0]
            err, n = masked_relerr(K, Kref, NBINS)
            assert np.all(K[Kref == 0.0] == 0.0)
            print(f"{case} precision {prec}: {err:.2e} over {n} points")
            assert err < tol


def test_empty_line_list():
    """No lines at all: K = kmin everywhere in both forms, the fit runs on it,
    and the adjoint returns zero gradients."""
    L = _lines([])
    kmin = 1e-30
    with _ctx(L) as ctx:
        assert ctx.num_lines == 0
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, CUT, kmin)
        for prec in (hkb.MIXED, hkb.PLAIN_FP64):
            K = ctx.opacity([T, 300.0], [P, 1e-3], prec)
            assert np.all(K == kmin)
        r = ctx.kdist(K[:1], nC=20)
        assert r["coeff"].shape == (1, NBINS, 20)
        dT, dP, dS, dG = ctx.opacity_vjp(T, P, np.ones(ctx.nx), hkb.MIXED)
        assert dT == 0.0 and dP == 0.0 and len(dS) == 0 and len(dG) == 0
