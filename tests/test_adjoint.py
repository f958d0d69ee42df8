"""GPU: the opacity adjoint (hk_opacity_vjp) against the FP64 oracle gradient
and central finite differences; the torch.autograd bridge.

Tolerances (written here): plain FP64 adjoint vs oracle 1e-9 relative;
mixed adjoint (regions A/B in FP32) vs oracle 1e-4 relative on dLoss/dT and
dLoss/dP and 1e-5 of the largest per-line value; finite differences (h = 1e-3
relative, central) vs the oracle gradient 1e-4 relative.
"""
import numpy as np
import pytest

import hkb
import oracle
from hkb import synth

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS = 1000.0, 1300.0, 0.01, 10
T0, P0 = 800.3, 1.0


@pytest.fixture(scope="module")
def adj():
    L = synth.hitran_lines(800, seed=5, nu_max=NUMAX, nu_min=NUMIN)
    Tq, Qq = synth.q_table()
    ctx = hkb.Context(0)
    ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
    ctx.set_partition(0, Tq, Qq)
    ctx.set_options(qalphaL=1.0)
    ctx.load_lines_hitran(L)
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    w = np.random.default_rng(0).standard_normal(ctx.nx)
    yield dict(ctx=ctx, L=L, Tq=Tq, Qq=Qq, w=w)
    ctx.close()


def loss(d, T, P, precision=hkb.PLAIN_FP64):
    K = d["ctx"].opacity([T], [P], precision)[0]
    return float(np.sum(d["w"] * np.log(K))), K


def reference(d, T=T0, P=P0, u=None):
    nx = d["ctx"].nx
    if u is None:
        u = d["w"] / loss(d, T, P)[1]
    return oracle.vjp_hitran(d["L"], synth.MASS, d["Tq"], d["Qq"], T, P, u, NUMIN, DNU, nx)


def test_vjp_plain_and_mixed_vs_oracle(adj):
    ctx = adj["ctx"]
    _, K = loss(adj, T0, P0)
    u = adj["w"] / K
    rT, rP, rS, rG = reference(adj, u=u)
    for prec, tol, tol_line in ((hkb.PLAIN_FP64, 1e-9, 1e-9), (hkb.MIXED, 1e-4, 1e-5)):
        dT, dP, dS, dG = ctx.opacity_vjp(T0, P0, u, prec)
        eT, eP = abs(dT - rT) / abs(rT), abs(dP - rP) / abs(rP)
        eS = np.max(np.abs(dS - rS)) / np.max(np.abs(rS))
        eG = np.max(np.abs(dG - rG)) / np.max(np.abs(rG))
        print(f"precision {prec}: dT {eT:.2e} dP {eP:.2e} dlogS {eS:.2e} dgammaL {eG:.2e}")
        assert eT < tol and eP < tol
        assert eS < tol_line and eG < tol_line


@pytest.mark.parametrize("case", ["beyond_fp32", "wide_tile"])
def test_vjp_mixed_seed_range(adj, case):
    """The mixed form stages u per 8192-point tile as FP32 scaled by a power
    of two; a seed beyond the FP32 range takes the scale, and a tile whose
    nonzero |u| span more than 2^64 keeps u and its sums in FP64."""
    ctx = adj["ctx"]
    _, K = loss(adj, T0, P0)
    u = adj["w"] / K
    if case == "beyond_fp32":
        u = u * 1e45
    else:
        u = u.copy()
        u[:5000] *= 1e30   # first tile only
        u[20000:20010] = 0.0
    rT, rP, rS, rG = reference(adj, u=u)
    dT, dP, dS, dG = ctx.opacity_vjp(T0, P0, u, hkb.MIXED)
    eT, eP = abs(dT - rT) / abs(rT), abs(dP - rP) / abs(rP)
    eS = np.max(np.abs(dS - rS)) / np.max(np.abs(rS))
    eG = np.max(np.abs(dG - rG)) / np.max(np.abs(rG))
    print(f"{case}: dT {eT:.2e} dP {eP:.2e} dlogS {eS:.2e} dgammaL {eG:.2e}")
    assert np.all(np.isfinite(dS)) and np.all(np.isfinite(dG))
    assert eT < 1e-4 and eP < 1e-4
    assert eS < 1e-5 and eG < 1e-5
    if case == "wide_tile":
        # lines of the other tiles, on their own scale
        far = np.zeros(ctx.num_lines, bool)
        far[ctx.line_order()] = ctx.state_lines(T0, P0)[0] > NUMIN + 5000 * DNU + 60.0
        m = np.max(np.abs(rS[far]))
        assert np.max(np.abs(dS[far] - rS[far])) < 1e-5 * m


@pytest.mark.parametrize("profile", [2, 3, 4])
def test_vjp_profiles_2_to_4(adj, profile):
    """Profiles 2-4: windows hold region A only, whose term is the profile's
    shape (Lorentz; Doppler and binned Gaussian in the FP64 form in both
    precisions, without y dependence and, for the binned Gaussian, with the
    grid step vb = dnu iad in the iad derivative).  Both precisions against
    the oracle gradient with the profile's windows, the plain one against
    central differences.  The Doppler and binned-Gaussian cores leave most
    grid points empty, so K carries a floor kmin (constant in every
    parameter) there."""
    ctx = adj["ctx"]
    ctx.set_profile(profile, 0)
    try:
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        kmin = 1e-12 * ctx.opacity([T0], [P0], hkb.PLAIN_FP64)[0].max()
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0, kmin)
        K = ctx.opacity([T0], [P0], hkb.PLAIN_FP64)[0]
        u = adj["w"] / K
        rT, rP, rS, rG = oracle.vjp_hitran(adj["L"], synth.MASS, adj["Tq"], adj["Qq"], T0, P0, u,
                                           NUMIN, DNU, ctx.nx, profile=profile)
        got = {}
        for prec, tol, tol_line in ((hkb.PLAIN_FP64, 1e-9, 1e-9), (hkb.MIXED, 1e-4, 1e-5)):
            dT, dP, dS, dG = got[prec] = ctx.opacity_vjp(T0, P0, u, prec)
            eT = abs(dT - rT) / abs(rT)
            eP = abs(dP - rP) / abs(rP) if rP != 0.0 else abs(dP)
            eS = np.max(np.abs(dS - rS)) / np.max(np.abs(rS))
            if profile == 2:
                eG = np.max(np.abs(dG - rG)) / np.max(np.abs(rG))
            else:
                assert np.all(rG == 0.0)
                eG = float(np.max(np.abs(dG)))
            print(f"profile {profile} precision {prec}: dT {eT:.2e} dP {eP:.2e} dlogS {eS:.2e} "
                  f"dgammaL {eG:.2e}")
            assert eT < tol and eP < tol
            assert eS < tol_line and eG < tol_line
        if profile >= 3:
            # the Doppler and binned-Gaussian adjoint runs its FP64 kernels in
            # either precision: the mixed request must give the plain result,
            # up to the order of the FP64 atomic additions
            _same_up_to_atomics(got[hkb.MIXED], got[hkb.PLAIN_FP64])
        dT, fT, dP, fP = _fd_vs_vjp(ctx, adj["w"], 800.5, P0)
        print(f"profile {profile}: dT {dT:.6g} fd {fT:.6g}; dP {dP:.6g} fd {fP:.6g}")
        assert abs(fT - dT) < 1e-5 * abs(dT)
        assert abs(fP - dP) <= 1e-5 * abs(dP)
    finally:
        ctx.set_profile(1, 0)
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)


def _same_up_to_atomics(a, b, rtol=1e-12):
    """Two VJP results of the same FP64 kernels: per-line sums are added with
    atomics, so only their order (the last bits) may differ."""
    for x, y in zip(a[:2], b[:2]):
        assert abs(x - y) <= rtol * abs(y) + 1e-300
    for x, y in zip(a[2:], b[2:]):
        m = np.max(np.abs(y))
        assert np.max(np.abs(x - y)) <= rtol * m + 1e-300


def test_vjp_doppler_cut_mode_1(adj):
    """Profile 3 with cutMode 1: the window half-width cut * gammaL moves with
    T and P, so the gradient holds the windows fixed (their edges are not
    differentiated).  Against the oracle gradient on the same windows, and
    against central differences taken with steps small enough that no window
    index changes (checked)."""
    ctx = adj["ctx"]
    cut = 500.0
    ctx.set_profile(3, 0)
    try:
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 1, cut)
        kmin = 1e-12 * ctx.opacity([T0], [P0], hkb.PLAIN_FP64)[0].max()
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 1, cut, kmin)
        K = ctx.opacity([T0], [P0], hkb.PLAIN_FP64)[0]
        u = adj["w"] / K
        rT, rP, rS, _ = oracle.vjp_hitran(adj["L"], synth.MASS, adj["Tq"], adj["Qq"], T0, P0, u,
                                          NUMIN, DNU, ctx.nx, cut=cut, profile=3, cutMode=1)
        got = {}
        for prec in (hkb.PLAIN_FP64, hkb.MIXED):
            dT, dP, dS, _ = got[prec] = ctx.opacity_vjp(T0, P0, u, prec)
            print(f"Doppler cutMode 1 precision {prec}: dT {dT:.6g} ref {rT:.6g}; dP {dP:.6g} "
                  f"ref {rP:.6g}")
            assert abs(dT - rT) < 1e-9 * abs(rT)
            assert (abs(dP - rP) / abs(rP) if rP != 0.0 else abs(dP)) < 1e-9
            assert np.max(np.abs(dS - rS)) < 1e-9 * np.max(np.abs(rS))
        _same_up_to_atomics(got[hkb.MIXED], got[hkb.PLAIN_FP64])
        win0 = ctx.state_lines(T0, P0)[4]

        def fixed_windows(T, P):
            return np.array_equal(ctx.state_lines(T, P)[4], win0)

        def lossf(T, P):
            return float(np.sum(adj["w"] * np.log(ctx.opacity([T], [P], hkb.PLAIN_FP64)[0])))
        # the largest relative step at which no window index moves
        for h in (1e-6, 1e-7, 1e-8, 1e-9):
            if all(fixed_windows(T0 * (1 + s), P0) and fixed_windows(T0, P0 * (1 + s))
                   for s in (h, -h)):
                break
        else:
            pytest.fail("every step moved a window index")
        hT, hP = h * T0, h * P0
        fT = (lossf(T0 + hT, P0) - lossf(T0 - hT, P0)) / (2 * hT)
        fP = (lossf(T0, P0 + hP) - lossf(T0, P0 - hP)) / (2 * hP)
        print(f"Doppler cutMode 1: step {h:g}, fd dT {fT:.6g}, fd dP {fP:.6g}")
        assert abs(fT - rT) < 1e-4 * abs(rT)
        # no pressure dependence inside fixed windows (delta = 0 here): the
        # difference quotient is rounding only
        assert abs(fP) <= 1e-4 * abs(fT) + 1e-12 * abs(lossf(T0, P0)) / hP
    finally:
        ctx.set_profile(1, 0)
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)


def test_vjp_vs_central_differences(adj):
    ctx = adj["ctx"]
    rT, rP, rS, rG = reference(adj)
    hT, hP = 1e-3 * T0, 1e-3 * P0
    fT = (loss(adj, T0 + hT, P0)[0] - loss(adj, T0 - hT, P0)[0]) / (2 * hT)
    fP = (loss(adj, T0, P0 + hP)[0] - loss(adj, T0, P0 - hP)[0]) / (2 * hP)
    print(f"dT {rT:.6g} fd {fT:.6g}; dP {rP:.6g} fd {fP:.6g}")
    assert abs(fT - rT) / abs(rT) < 1e-4
    assert abs(fP - rP) / abs(rP) < 1e-4
    # per line: strength and width multipliers of the two lines with the
    # largest gradients, through hk_set_line_scales
    n = ctx.num_lines
    _, _, iad, vy, _ = ctx.state_lines(T0, P0)
    aL = np.empty(n)
    aL[ctx.line_order()] = vy / iad
    e = 1e-3
    for l in np.argsort(-np.abs(rS))[:2]:
        s = np.ones(n)
        s[l] = np.exp(e)
        ctx.set_line_scales(s, None)
        lp = loss(adj, T0, P0)[0]
        s[l] = np.exp(-e)
        ctx.set_line_scales(s, None)
        lm = loss(adj, T0, P0)[0]
        assert abs((lp - lm) / (2 * e) - rS[l]) < 1e-4 * abs(rS[l])
    for l in np.argsort(-np.abs(rG * aL))[:2]:
        gsc = np.ones(n)
        gsc[l] = np.exp(e)
        ctx.set_line_scales(None, gsc)
        lp = loss(adj, T0, P0)[0]
        gsc[l] = np.exp(-e)
        ctx.set_line_scales(None, gsc)
        lm = loss(adj, T0, P0)[0]
        assert abs((lp - lm) / (2 * e) - rG[l] * aL[l]) < 1e-4 * abs(rG[l] * aL[l])
    ctx.set_line_scales(None, None)


def test_autograd_function(adj):
    import torch
    from hkb.autograd import Opacity
    ctx = adj["ctx"]
    n = ctx.num_lines
    T = torch.tensor(T0, dtype=torch.float64, requires_grad=True)
    P = torch.tensor(P0, dtype=torch.float64, requires_grad=True)
    log_s = torch.zeros(n, dtype=torch.float64, requires_grad=True)
    log_g = torch.zeros(n, dtype=torch.float64, requires_grad=True)
    w = torch.as_tensor(adj["w"], device="cuda")
    K = Opacity.apply(ctx, T, P, log_s, log_g, hkb.PLAIN_FP64)
    L = torch.sum(w * torch.log(K))
    L.backward()
    rT, rP, rS, rG = reference(adj)
    _, _, iad, vy, _ = ctx.state_lines(T0, P0)
    aL = np.empty(n)
    aL[ctx.line_order()] = vy / iad
    assert abs(T.grad.item() - rT) < 1e-9 * abs(rT)
    assert abs(P.grad.item() - rP) < 1e-9 * abs(rP)
    assert np.max(np.abs(log_s.grad.numpy() - rS)) < 1e-9 * np.max(np.abs(rS))
    assert np.max(np.abs(log_g.grad.numpy() - rG * aL)) < 1e-9 * np.max(np.abs(rG * aL))
    ctx.set_line_scales(None, None)


def _fd_vs_vjp(ctx, w, T0, P0, h=2.5e-4):
    """dLoss/dT, dLoss/dP of Loss = sum w log K from the VJP (plain FP64)
    against central differences of the forward at h and h/2 relative,
    Richardson-extrapolated (error O(h^4): the net derivative can be a small
    difference of large per-line terms).  T0 +- h T0 must stay inside one
    segment of the partition table (1 K nodes): Q(T) is piecewise linear and
    the VJP takes the slope of the segment holding T0."""
    def lossf(T, P):
        return float(np.sum(w * np.log(ctx.opacity([T], [P], hkb.PLAIN_FP64)[0])))

    def central(dT_, dP_):
        if dT_:
            return (lossf(T0 + dT_, P0) - lossf(T0 - dT_, P0)) / (2 * dT_)
        return (lossf(T0, P0 + dP_) - lossf(T0, P0 - dP_)) / (2 * dP_)
    K = ctx.opacity([T0], [P0], hkb.PLAIN_FP64)[0]
    assert np.all(K > 0.0)
    dT, dP, _, _ = ctx.opacity_vjp(T0, P0, w / K, hkb.PLAIN_FP64)
    hT, hP = h * T0, h * P0
    fT = (4.0 * central(hT / 2, 0) - central(hT, 0)) / 3.0
    fP = (4.0 * central(0, hP / 2) - central(0, hP)) / 3.0
    return dT, fT, dP, fP


def test_vjp_exomol_vs_central_differences():
    """ExoMol lists: S scaling by exp(-c2 E''/T) without the HITRAN
    reference-temperature ratio, widths from the species defaults with P0 =
    1 bar; the chain rule of adjoint_line_kernel's ExoMol branch."""
    L = synth.exomol_lines(3000, seed=8, nu_max=NUMAX)
    L["nu"] = NUMIN - 30.0 + (NUMAX - NUMIN + 60.0) * (L["nu"] / NUMAX)
    Tq, Qq = synth.q_table()
    with hkb.Context(0) as ctx:
        ctx.set_species(hkb.EXOMOL, [synth.MASS], [1.0], defaultL=0.07, defaultn=0.5)
        ctx.set_partition(0, Tq, Qq)
        ctx.load_lines_exomol(L)
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        w = np.random.default_rng(3).standard_normal(ctx.nx)
        dT, fT, dP, fP = _fd_vs_vjp(ctx, w, 800.5, P0)
    print(f"exomol: dT {dT:.6g} fd {fT:.6g}; dP {dP:.6g} fd {fP:.6g}")
    assert abs(fT - dT) < 1e-4 * abs(dT)
    assert abs(fP - dP) < 1e-4 * abs(dP)


def test_vjp_two_isotopologues_vs_central_differences():
    """Two isotopologues with their own masses, abundances and partition
    tables: d ln Q / dT per isotopologue in the chain rule."""
    L = synth.hitran_lines(1500, seed=9, nu_max=NUMAX + 30.0, nu_min=NUMIN - 30.0)
    L["iso"] = (np.arange(1500) % 3 == 0).astype(np.int32)
    L["delta"] = np.random.default_rng(4).uniform(-0.01, 0.01, 1500)
    Tq, Qq = synth.q_table()
    with hkb.Context(0) as ctx:
        ctx.set_species(hkb.HITRAN, [synth.MASS, synth.MASS + 2.0], [0.9, 0.1])
        ctx.set_partition(0, Tq, Qq)
        ctx.set_partition(1, Tq, Qq * (1.0 + Tq / 3000.0))
        ctx.set_options(qalphaL=0.6)
        ctx.load_lines_hitran(L)
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        w = np.random.default_rng(5).standard_normal(ctx.nx)
        dT, fT, dP, fP = _fd_vs_vjp(ctx, w, 800.5, P0)
    print(f"two isotopologues: dT {dT:.6g} fd {fT:.6g}; dP {dP:.6g} fd {fP:.6g}")
    assert abs(fT - dT) < 1e-4 * abs(dT)
    assert abs(fP - dP) < 1e-4 * abs(dP)
