"""The per-line index windows equal a brute-force evaluation of the FP64
cutoff / region predicates at every grid point (all cut modes)."""
import numpy as np
import pytest

import oracle
from hkb import synth


@pytest.mark.parametrize("T,P,cut,mode", [
    (1500.0, 0.1, 25.0, 0), (300.0, 1e-6, 25.0, 0), (2000.0, 100.0, 10.0, 0),
    (800.0, 1.0, 5.0, 1), (800.0, 1.0, 50.0, 2), (1000.0, 1.0, 0.0, 0)])
def test_windows_brute_force(T, P, cut, mode):
    L = synth.hitran_lines(2000, seed=5, nu_max=2000.0)
    Tq, Qq = synth.q_table()
    Q = oracle.partition(Tq, Qq, T)
    nu, S, iad, vy = oracle.prep_hitran(L, [18.0], [1.0], [Q], T, P)
    numin, dnu = 0.0, 0.01
    nx = oracle.grid_nx(0.0, 2000.0, dnu)
    win = oracle.windows(nu, S, iad, vy, numin, dnu, nx, mode, cut)
    x = oracle.grid_x(numin, dnu, nx)
    idx = np.arange(nx)
    cutv = 1e30 if cut == 0 else cut
    for l in np.random.default_rng(1).choice(len(nu), 150, replace=False):
        d = x - nu[l]
        w = cutv if mode == 0 else (cutv * vy[l] / iad[l] if mode == 1 else cutv / iad[l])
        inw = np.abs(d) < w
        xx = d * iad[l]
        r2 = xx * xx + vy[l] * vy[l]
        i0, b0, c0, c1, b1, i1 = win[l]
        assert np.array_equal(inw, (idx >= i0) & (idx < i1))
        assert np.array_equal(inw & (r2 < 1e6), (idx >= b0) & (idx < b1))
        assert np.array_equal(inw & (r2 < 100), (idx >= c0) & (idx < c1))


def test_zero_strength_lines_have_empty_windows():
    L = synth.hitran_lines(50, seed=2, nu_max=100.0)
    L["nu"][:5] = 0.0          # S2_kernel zeroes lines at nu == 0
    L["S"][5:10] = 0.0
    Tq, Qq = synth.q_table()
    nu, S, iad, vy = oracle.prep_hitran(L, [18.0], [1.0], [oracle.partition(Tq, Qq, 500.0)],
                                        500.0, 1.0)
    win = oracle.windows(nu, S, iad, vy, 0.0, 0.01, 10000, 0, 25.0)
    assert np.all(win[:10, 5] == win[:10, 0])
    assert np.all(win[10:, 5] > win[10:, 0])
