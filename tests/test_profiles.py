"""GPU: profiles 2-4 and plinth removal (hk_set_profile) against the FP64
oracle (voigt.h:1091-1262 restated).

The mixed form runs when the mixed precision is asked for -- the Voigt and
Lorentz profiles with sub-Lorentzian wings or plinth removal, the Doppler
profile with plinth removal, the binned Gaussian (FP32 where their terms are
normal floats, FP64 tails beyond): 1e-5 relative where K > 1e-6 of its bin maximum (the mixed
bound), and faster than the FP64 form.  Plinth removal in the mixed form
takes profile - plinth without cancellation (factored differences, or FP64
per point for lines whose cut edge lies in region C or near a region
boundary); sub-Lorentzian wings with plinth removal run the FP64 form, whose
bound for differences of profile values and plinths is 1e-9; the FP64 form
itself: 1e-12.  Index windows (no regions B and C for profiles 2-4) are
bit-exact.
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
            ctx.opacity([T], [P], prec)  # time a warm call: the first may load the kernel
            ms[prec] = ctx.last_timing()[0]
            err, n = masked_relerr(K, Kref, NBINS)
            print(f"profile {profile} plinth {plinth} cut {cutMode}/{cut} T={T} P={P} "
                  f"precision {prec}: err {err:.2e}, line sum {ms[prec]:.3f} ms")
            if prec == hkb.MIXED:
                assert err < 1e-5
            else:
                assert err < (1e-9 if plinth else 1e-12)
        # the mixed form saves per-pair work; with windows of a few points
        # (the 0.05 cm^-1 Doppler cut) per-tile costs decide either form
        if ms[hkb.PLAIN_FP64] > 0.2:
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
                ctx.opacity([T], [P], prec)  # time a warm call
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
                                                 (2, 0, True), (1, 1, False), (2, 1, False),
                                                 (3, 1, False)])
def test_profile_tables_equal_opacity(small, profile, plinth, subl):
    """The mixed kernels of the Gaussian profiles, of sub-Lorentzian wings and
    of plinth removal in both table modes (per-batch launches and one persistent launch) give
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


# Plinth removal with cut edges in bins of their own: 60 lines over 12
# decades of strength, 10 cm^-1 bins, so most bins hold one or two windows
# and K at a point beside a cut edge is that line's profile - plinth alone
# (the plain FP32 difference misses 1e-5 there by orders of magnitude).  The
# cut rules put the edges in every class: r_c^2 = x_c^2 + y^2 below 400 and
# within a factor 4 of r^2 = 1e6 (FP64 per point), in region B and in
# region A (factored differences).
SPARSE_BINS = 300
EDGE_CASES = [(1, 0, 25.0), (1, 1, 300.0), (1, 1, 3.0), (1, 2, 15.0), (1, 2, 100.0),
              (1, 2, 1500.0), (1, 2, 5000.0), (2, 0, 25.0), (2, 1, 50.0), (3, 2, 4.0),
              (3, 0, 0.03)]


@pytest.fixture(scope="module")
def sparse():
    L = synth.hitran_lines(60, seed=5, nu_max=3000.0)
    Tq, Qq = synth.q_table()
    ctx = hkb.Context(0)
    ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
    ctx.set_partition(0, Tq, Qq)
    ctx.set_options(qalphaL=1.0)
    ctx.load_lines_hitran(L)
    yield dict(ctx=ctx, L=L, Tq=Tq, Qq=Qq)
    ctx.set_profile(1, 0)
    ctx.close()


@pytest.mark.parametrize("profile,cutMode,cut", EDGE_CASES)
def test_plinth_isolated_edges(sparse, profile, cutMode, cut):
    ctx = sparse["ctx"]
    ctx.set_profile(profile, 1)
    ctx.set_grid(NUMIN, NUMAX, DNU, SPARSE_BINS, cutMode, cut)
    try:
        total = 0
        for T, P in ((1500.0, 0.1), (500.0, 10.0), (2500.0, 1e-3)):
            Kref, _ = oracle_k(sparse, T, P, profile, 1, cutMode, cut)
            K = ctx.opacity([T], [P], hkb.MIXED)[0]
            if not (Kref > 0).any():
                # windows narrower than a grid step (a cut of a few Lorentz
                # widths at low pressure): nothing to compare but zeros
                assert np.abs(K - Kref).max() <= 1e-5 * max(np.abs(Kref).max(), 1e-300)
                continue
            err, n = masked_relerr(K, Kref, SPARSE_BINS)
            total += n
            print(f"isolated edges: profile {profile} cut {cutMode}/{cut} T={T} P={P}: "
                  f"err {err:.2e} over {n} points")
            assert err < 1e-5
        assert total > 0
    finally:
        ctx.set_profile(1, 0)
