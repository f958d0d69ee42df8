"""GPU: profiles 2-4 and plinth removal (hk_set_profile) against the FP64
oracle (voigt.h:1091-1262 restated).

The mixed form runs when the mixed precision is asked for -- the Voigt and
Lorentz profiles with and without sub-Lorentzian wings, the Doppler and
binned-Gaussian profiles (where their FP32 terms are normal floats): 1e-5
relative where K > 1e-6 of its bin maximum (the mixed bound), and faster
than the FP64 form.  Plinth removal runs the FP64 form in both precisions
(profile - plinth cancels near window edges), so its bound is the FP64 one
for differences of profile values and plinths: 1e-9; the FP64 form itself:
1e-12.  Index windows (no regions B and C for profiles 2-4) are bit-exact.
"""
import numpy as np
import pytest

import hkb
import oracle
from hkb import synth
from test_gpu_parity import NBINS, DNU, NUMAX, NUMIN, masked_relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    L = synth.hitran_lines(20000, seed=11, nu_max=3000.0)
    Tq, Qq = synth.q_table()
    ctx = hkb.Context(0)
    ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
    ctx.set_partition(0, Tq, Qq)
    ctx.set_options(qalphaL=1.0)
    ctx.load_lines_hitran(L)
    yield dict(ctx=ctx, L=L, Tq=Tq, Qq=Qq)
    ctx.set_profile(1, 0)
    ctx.close()


def oracle_k(d, T, P, profile, plinth, cutMode, cut):
    Q = oracle.partition(d["Tq"], d["Qq"], T)
    nu, S, iad, vy = oracle.prep_hitran(d["L"], [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, cutMode, cut, profile=profile)
    pl = oracle.plinth(S, iad, vy, win, cutMode, cut, profile) if plinth else None
    K, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx, profile=profile, plinth=pl)
    return K, win


CASES = [(2, 0, 0, 25.0), (3, 0, 0, 25.0), (4, 0, 0, 25.0), (2, 0, 1, 500.0), (3, 0, 2, 40.0),
         (1, 1, 0, 25.0), (2, 1, 0, 10.0), (3, 1, 0, 0.05), (1, 1, 1, 300.0)]


@pytest.mark.parametrize("profile,plinth,cutMode,cut", CASES)
def test_profile_matches_oracle(small, profile, plinth, cutMode, cut):
    ctx = small["ctx"]
    ctx.set_profile(profile, plinth)
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, cutMode, cut)
    for T, P in ((1500.0, 0.1), (500.0, 10.0)):
        Kref, win = oracle_k(small, T, P, profile, plinth, cutMode, cut)
        # the index rule on the device's own FP64 line parameters, bit-exact
        gnu, gS, giad, gvy, gwin = ctx.state_lines(T, P)
        nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
        assert np.array_equal(gwin, oracle.windows(gnu, gS, giad, gvy, NUMIN, DNU, nx, cutMode, cut,
                                                   profile=profile))
        if profile != 1:
            assert np.all(gwin[:, 1] == gwin[:, 2]) and np.all(gwin[:, 3] == gwin[:, 4])
        ms = {}
        for prec in (hkb.MIXED, hkb.PLAIN_FP64):
            K = ctx.opacity([T], [P], prec)[0]
            ms[prec] = ctx.last_timing()[0]
            err, n = masked_relerr(K, Kref, NBINS)
            print(f"profile {profile} plinth {plinth} cut {cutMode}/{cut} T={T} P={P} "
                  f"precision {prec}: err {err:.2e}, line sum {ms[prec]:.3f} ms")
            if prec == hkb.MIXED and not plinth:
                assert err < 1e-5
            else:
                assert err < (1e-9 if plinth else 1e-12)
        if not plinth:
            assert ms[hkb.MIXED] < ms[hkb.PLAIN_FP64]
    if not plinth:
        ctx.opacity_vjp(1500.0, 0.1, np.ones(ctx.nx))  # every profile has an adjoint
    else:
        with pytest.raises(hkb.HkError) as e:
            ctx.opacity_vjp(1500.0, 0.1, np.ones(ctx.nx))
        assert e.value.status == -8
    ctx.set_profile(1, 0)


def test_profile_arguments(small):
    ctx = small["ctx"]
    for bad in ((0, 0), (5, 0), (1, 2)):
        with pytest.raises(hkb.HkError) as e:
            ctx.set_profile(*bad)
        assert e.value.status == -1


SL14 = [3.0, 10.0, 20.0, 0.09, -0.05, 0.004, 0.05, 0.02, 0.003, 0.02, 0.0, 0.0, 1100.0, 2900.0]


@pytest.mark.parametrize("profile,plinth", [(1, 0), (2, 0), (1, 1)])
def test_sublorentzian_matches_oracle(small, profile, plinth):
    ctx = small["ctx"]
    ctx.set_profile(profile, plinth)
    ctx.set_sublorentzian(SL14)
    try:
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        for T, P in ((1500.0, 0.1), (500.0, 10.0)):
            Q = oracle.partition(small["Tq"], small["Qq"], T)
            nu, S, iad, vy = oracle.prep_hitran(small["L"], [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
            nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
            win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, 25.0, profile=profile)
            pl = oracle.plinth(S, iad, vy, win, 0, 25.0, profile) if plinth else None
            Kref, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx, profile=profile, plinth=pl,
                                     sublorentz=oracle.sublorentz_params(SL14, T))
            ms = {}
            for prec in (hkb.MIXED, hkb.PLAIN_FP64):
                K = ctx.opacity([T], [P], prec)[0]
                ms[prec] = ctx.last_timing()[0]
                err, _ = masked_relerr(K, Kref, NBINS)
                print(f"sub-Lorentzian profile {profile} plinth {plinth} T={T} precision {prec}: "
                      f"err {err:.2e}, line sum {ms[prec]:.3f} ms")
                if prec == hkb.MIXED and not plinth:
                    assert err < 1e-5
                else:
                    assert err < (1e-9 if plinth else 1e-12)
            if not plinth:
                assert ms[hkb.MIXED] < ms[hkb.PLAIN_FP64]
    finally:
        ctx.set_sublorentzian(None)
        ctx.set_profile(1, 0)
    with pytest.raises(hkb.HkError) as e:
        ctx.set_profile(4, 1)  # heliosk.cu:410-413
    assert e.value.status == -8


@pytest.mark.parametrize("profile,plinth,subl", [(3, 0, False), (4, 0, False), (1, 0, True),
                                                 (2, 0, True)])
def test_profile_tables_equal_opacity(small, profile, plinth, subl):
    """The mixed kernels of the Gaussian profiles and of sub-Lorentzian wings
    in both table modes (per-batch launches and one persistent launch) give
    the same bits as hk_opacity."""
    import torch
    ctx = small["ctx"]
    ctx.set_profile(profile, plinth)
    if subl:
        ctx.set_sublorentzian(SL14)
    try:
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        Ts = np.array([1500.0, 500.0, 900.0, 2200.0, 300.0])
        Ps = np.array([0.1, 10.0, 1.0, 1e-3, 0.5])
        ref = ctx.opacity(Ts, Ps, hkb.MIXED)
        ns, nx = len(Ts), ctx.nx
        K = torch.empty((ns, nx), dtype=torch.float64, device="cuda")
        coeff = torch.empty((ns, NBINS, 20), dtype=torch.float64, device="cuda")
        nxmin = torch.empty((ns, NBINS), dtype=torch.int32, device="cuda")
        for mode in (0, 1):
            ctx.set_table_mode(mode)
            ctx.table_build(Ts, Ps, K, coeff, nxmin, nC=20)
            assert ctx.table_kernels == (2 if mode else 4)
            ctx.table_run()
            ctx.table_status()
            assert np.array_equal(K.cpu().numpy(), ref), f"table mode {mode}"
            ctx.table_free()
    finally:
        ctx.set_table_mode(0)
        ctx.set_sublorentzian(None)
        ctx.set_profile(1, 0)
