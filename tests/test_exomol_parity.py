"""GPU parity of the ExoMol forward path: the line scaling of L_kernelExomol
(voigt.h:484-504) + Sf_kernel (voigt.h:365-397, called with c1 = h c / (kB T)
and T1 = T0 / T, heliosk.cu:985-986, 1100) and the Voigt sum, through the
C ABI, against the FP64 oracle (oracle.prep_exomol + oracle.opacity).

Lines follow the ExoMol-scale workload's distributions on a slice: nu0 ~
U[0, 40000] mapped onto 0-3000 cm^-1 (+- 30 cm^-1 beyond the grid ends),
log10 S ~ U[-40, -18], E'' ~ Exp(8000), gamma_L = 0.07 and n = 0.5 from the
species defaults, a nonzero Einstein-A column (natural width A / (4 pi c)),
pressure in bar (P0 = 1 bar for ExoMol), two states.

Tolerances (written here): nu exact, 1/alphaD 2e-16, S and y 1e-14 relative
(one FP64 exp each, device vs host libm); windows bit-exact; K 1e-12 (plain
FP64 form) and 1e-5 (mixed form) relative where K > 1e-6 of its bin maximum.
"""
import numpy as np
import pytest

import hkb
import oracle
from hkb import synth

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS, CUT = 0.0, 3000.0, 0.01, 30, 25.0
DEFAULT_L, DEFAULT_N = 0.07, 0.5
STATES = [(500.0, 1e-4), (2500.0, 10.0)]


@pytest.fixture(scope="module")
def exo():
    L = synth.exomol_lines(20000, seed=31)
    L["nu"] = (NUMIN - 30.0) + (NUMAX - NUMIN + 60.0) * (L["nu"] / 40000.0)
    L["A"] = np.random.default_rng(32).uniform(0.0, 50.0, len(L["nu"]))
    Tq, Qq = synth.q_table()
    ctx = hkb.Context(0)
    ctx.set_species(hkb.EXOMOL, [synth.MASS], [1.0], defaultL=DEFAULT_L, defaultn=DEFAULT_N)
    ctx.set_partition(0, Tq, Qq)
    ctx.load_lines_exomol(L)
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, CUT)
    yield dict(ctx=ctx, L=L, Tq=Tq, Qq=Qq, order=ctx.line_order())
    ctx.close()


def oracle_state(d, T, P):
    Q = oracle.partition(d["Tq"], d["Qq"], T)
    nu, S, iad, vy = oracle.prep_exomol(d["L"], synth.MASS, 1.0, Q, DEFAULT_L, DEFAULT_N, T, P)
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, CUT)
    return nu, S, iad, vy, win


def masked_relerr(K, Kref):
    Kr = Kref.reshape(NBINS, -1)
    Kg = K.reshape(NBINS, -1)
    mask = Kr > 1e-6 * Kr.max(axis=1, keepdims=True)
    return float((np.abs(Kg[mask] - Kr[mask]) / Kr[mask]).max()), int(mask.sum())


@pytest.mark.parametrize("T,P", STATES)
def test_exomol_state_lines_and_windows(exo, T, P):
    ctx, o = exo["ctx"], exo["order"]
    nu, S, iad, vy, win = ctx.state_lines(T, P)
    onu, oS, oiad, ovy, owin = (a[o] for a in oracle_state(exo, T, P))
    assert np.array_equal(nu, onu)
    assert np.allclose(iad, oiad, rtol=2e-16, atol=0)
    assert np.allclose(S, oS, rtol=1e-14, atol=0)
    assert np.allclose(vy, ovy, rtol=1e-14, atol=0)
    # the natural width is in y: widths differ from defaultL alone
    assert np.ptp(vy / np.where(iad > 0, iad, 1.0)) > 0
    assert np.array_equal(win, owin)


def test_exomol_opacity_plain_and_mixed(exo):
    ctx = exo["ctx"]
    Ts = [T for T, _ in STATES]
    Ps = [P for _, P in STATES]
    Kp = ctx.opacity(Ts, Ps, hkb.PLAIN_FP64)
    Km = ctx.opacity(Ts, Ps, hkb.MIXED)
    nx = ctx.nx
    for s, (T, P) in enumerate(STATES):
        nu, S, iad, vy, win = oracle_state(exo, T, P)
        Kref, pairs = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx)
        ep, n = masked_relerr(Kp[s], Kref)
        em, _ = masked_relerr(Km[s], Kref)
        print(f"ExoMol T={T} P={P} bar pairs(A,B,C)={pairs}: plain {ep:.2e} mixed {em:.2e} "
              f"over {n} points")
        assert ep < 1e-12
        assert em < 1e-5
