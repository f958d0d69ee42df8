"""GPU parity: libhkb's CUDA path (through the C ABI) against the FP64 oracle.

Tolerances (written here, stated by the build target):
  * window / region / bin indexing and per-bin sorted values: bit-exact;
  * plain FP64 form: 1e-12 relative where K > 1e-6 of its bin maximum;
  * mixed FP32/FP64 form: 1e-5 relative where K > 1e-6 of its bin maximum;
  * Chebyshev coefficients: 1e-9 absolute on identical K input, 1e-6
    absolute end to end from the mixed form.
"""
import numpy as np
import pytest

import hkb
import oracle
from hkb import synth

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS = 0.0, 3000.0, 0.01, 30
STATES = [(1500.0, 0.1), (300.0, 1e-6), (2000.0, 100.0), (1000.0, 1.0)]


@pytest.fixture(scope="module")
def small():
    """20000 synthetic lines on 0-3000 cm^-1 (a 1/10-scale 'small' workload)."""
    L = synth.hitran_lines(20000, seed=11, nu_max=3000.0)
    Tq, Qq = synth.q_table()
    ctx = hkb.Context(0)
    ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
    ctx.set_partition(0, Tq, Qq)
    ctx.set_options(qalphaL=1.0)
    ctx.load_lines_hitran(L)
    yield dict(ctx=ctx, L=L, Tq=Tq, Qq=Qq, order=ctx.line_order())
    ctx.close()


def oracle_state(d, T, P, cut=25.0, mode=0, irange=None):
    Q = oracle.partition(d["Tq"], d["Qq"], T)
    nu, S, iad, vy = oracle.prep_hitran(d["L"], [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, mode, cut)
    K, pairs = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx, irange=irange)
    return K, pairs, (nu, S, iad, vy, win)


def masked_relerr(K, Kref, nbins):
    Kr = Kref.reshape(nbins, -1)
    Kg = K.reshape(nbins, -1)
    mask = Kr > 1e-6 * Kr.max(axis=1, keepdims=True)
    err = np.abs(Kg[mask] - Kr[mask]) / np.abs(Kr[mask])
    return float(err.max()), int(mask.sum())


def test_profile_fp64_and_fp32(small):
    ctx = small["ctx"]
    rng = np.random.default_rng(3)
    r = 10 * np.sqrt(rng.random(20000))
    th = rng.random(20000) * np.pi / 2
    x, y = r * np.cos(th), r * np.sin(th)
    y[:5000] = 10 ** rng.uniform(-9, 0, 5000)
    x[5000:6000] = 0.0
    # the FP32 form switches from Algorithm 916 to the asymptotic series at
    # r = 6: both sides of the switch, and tiny y where the exp(-x^2) term
    # of the real axis dominates
    r6 = rng.uniform(5.9, 6.1, 2000)
    x[6000:8000], y[6000:8000] = r6 * np.cos(th[6000:8000]), r6 * np.sin(th[6000:8000])
    x[8000:9000] = rng.uniform(5.9, 10.0, 1000)
    y[8000:9000] = 10 ** rng.uniform(-12, 0, 1000)
    keep = x * x + y * y < 100
    x, y = x[keep], y[keep]
    ref = np.array([oracle.voigt916(a, b) for a, b in zip(x, y)])
    d64 = ctx.profile_eval(x, y, hkb.PLAIN_FP64)
    d32 = ctx.profile_eval(x, y, hkb.MIXED)
    e64 = np.max(np.abs(d64 - ref) / ref)
    # the FP32 form sees x, y rounded to float: compare against the oracle at
    # those rounded arguments so only the profile evaluation is measured
    xr, yr = x.astype(np.float32).astype(np.float64), y.astype(np.float32).astype(np.float64)
    ref32 = np.array([oracle.voigt916(a, b) for a, b in zip(xr, yr)])
    e32 = np.max(np.abs(d32 - ref32) / ref32)
    print(f"profile max rel err: fp64 {e64:.3e}  fp32 {e32:.3e}")
    assert e64 < 1e-12
    assert e32 < 2e-6


@pytest.mark.parametrize("T,P", STATES)
def test_state_lines_and_windows_bit_exact(small, T, P):
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    nu, S, iad, vy, win = ctx.state_lines(T, P)
    o = small["order"]
    _, _, (onu, oS, oiad, ovy, owin) = oracle_state(small, T, P, irange=(0, 1))
    onu, oS, oiad, ovy, owin = onu[o], oS[o], oiad[o], ovy[o], owin[o]
    assert np.array_equal(nu, onu)
    assert np.allclose(iad, oiad, rtol=2e-16, atol=0)
    assert np.allclose(S, oS, rtol=1e-14, atol=0)
    assert np.allclose(vy, ovy, rtol=1e-14, atol=0)
    # the index rule is bit-exact on identical FP64 line parameters ...
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    assert np.array_equal(win, oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, 25.0))
    # ... and, in practice, identical to the oracle's own prep
    assert np.array_equal(win, owin)


@pytest.mark.parametrize("T,P", STATES)
def test_opacity_plain_and_mixed(small, T, P):
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    Kref, pairs, _ = oracle_state(small, T, P)
    Kp = ctx.opacity([T], [P], hkb.PLAIN_FP64)[0]
    Km = ctx.opacity([T], [P], hkb.MIXED)[0]
    ep, n = masked_relerr(Kp, Kref, NBINS)
    em, _ = masked_relerr(Km, Kref, NBINS)
    print(f"T={T} P={P} pairs(A,B,C)={pairs} plain {ep:.2e} mixed {em:.2e} over {n} pts")
    assert ep < 1e-12
    assert em < 1e-5


@pytest.mark.parametrize("mode,cut", [(1, 50.0), (2, 30.0), (0, 0.0)])
def test_opacity_cut_modes(small, mode, cut):
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, mode, cut)
    T, P = 1200.0, 0.5
    Kref, pairs, _ = oracle_state(small, T, P, cut=cut, mode=mode)
    Km = ctx.opacity([T], [P], hkb.MIXED)[0]
    Kp = ctx.opacity([T], [P], hkb.PLAIN_FP64)[0]
    assert masked_relerr(Kp, Kref, NBINS)[0] < 1e-12
    assert masked_relerr(Km, Kref, NBINS)[0] < 1e-5


def test_opacity_fine_grid_unsplit_tiles(small):
    """A grid of >= 4736 tiles runs every tile as one ticket; the 300000-point
    grid of the other tests splits each tile's line range into 8 parts whose
    sums are combined in part order.  Both must match the oracle."""
    ctx = small["ctx"]
    numin, numax, dnu, nbins = 0.0, 1000.0, 1e-4, 10
    ctx.set_grid(numin, numax, dnu, nbins, 0, 25.0)
    nx = ctx.nx
    assert nx == oracle.grid_nx(numin, numax, dnu)
    assert -(-nx // hkb.tile_points()) >= 4736
    T, P = 1500.0, 0.1
    Km = ctx.opacity([T], [P], hkb.MIXED)[0]
    Kp = ctx.opacity([T], [P], hkb.PLAIN_FP64)[0]
    Q = oracle.partition(small["Tq"], small["Qq"], T)
    nu, S, iad, vy = oracle.prep_hitran(small["L"], [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    win = oracle.windows(nu, S, iad, vy, numin, dnu, nx, 0, 25.0)
    for ib in (0, 4_000_000 + 777, nx - 20000):
        Kr, _ = oracle.opacity(nu, S, iad, vy, win, numin, dnu, nx, irange=(ib, ib + 20000))
        sl = slice(ib, ib + 20000)
        mask = Kr > 1e-6 * Kr.max()
        ep = np.max(np.abs(Kp[sl] - Kr)[mask] / Kr[mask])
        em = np.max(np.abs(Km[sl] - Kr)[mask] / Kr[mask])
        print(f"fine grid [{ib}, +20000): plain {ep:.2e} mixed {em:.2e}")
        assert ep < 1e-12
        assert em < 1e-5


def test_opacity_extreme_strength_range():
    """Strengths over 270 decades: the mixed form sums each 2^96 band of line
    strengths ('level') in FP32 with its own power-of-two scale, and lines
    more than 2^768 below the strongest in FP64; lines near nu = 0 (tiny
    Doppler width, huge x) also take the FP64 path.  All must match the
    oracle."""
    L = synth.hitran_lines(6000, seed=21, logS=(-290.0, -18.0), nu_max=3000.0)
    L["nu"][:3] = [1e-3, 0.05, 2.0]
    Tq, Qq = synth.q_table()
    T, P = 900.0, 0.3
    with hkb.Context(0) as ctx:
        ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
        ctx.set_partition(0, Tq, Qq)
        ctx.set_options(qalphaL=1.0)
        ctx.load_lines_hitran(L)
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        Km = ctx.opacity([T], [P], hkb.MIXED)[0]
    Q = oracle.partition(Tq, Qq, T)
    nu, S, iad, vy = oracle.prep_hitran(L, [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, 25.0)
    Kr, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx)
    term = S * vy / np.pi / np.maximum(100.0, vy * vy)
    print("decades of line terms:", np.log10(term.max() / term[term > 0].min()))
    em, n = masked_relerr(Km, Kr, NBINS)
    # every point, not only those above 1e-6 of their bin maximum
    pos = Kr > 1e-280  # clear of FP64 subnormals
    eall = np.max(np.abs(Km[pos] - Kr[pos]) / Kr[pos])
    print(f"extreme range: mixed {em:.2e} over {n} pts, all points {eall:.2e}")
    assert em < 1e-5
    assert eall < 1e-5


def test_batched_states_equal_single_states(small):
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    Ts = np.array([s[0] for s in STATES])
    Ps = np.array([s[1] for s in STATES])
    Kb = ctx.opacity(Ts, Ps, hkb.MIXED)
    for s, (T, P) in enumerate(STATES):
        Ks = ctx.opacity([T], [P], hkb.MIXED)[0]
        assert np.array_equal(Kb[s], Ks)


def test_kdist_p004_golden(golden_p004):
    g = golden_p004
    with hkb.Context(0) as ctx:
        ctx.set_grid(0.0, 30000.0, 1.0, 1, 0, 25.0, 0.0)
        r = ctx.kdist(g["K_i"][None, :], nC=20, sorted_K=True)
        assert np.array_equal(r["sorted"][0], g["Ksorted_i"])
        r = ctx.kdist(g["K_r"][None, :], nC=20, recon=True)
        assert r["nxmin"][0, 0] == 4533
        assert np.max(np.abs(r["coeff"][0, 0] - g["cbin_r"][2:])) < 1e-9
        R = g["Krecon_r"]
        nz = R != 0
        assert np.array_equal(r["recon"][0][~nz], R[~nz])
        assert np.max(np.abs(r["recon"][0][nz] - R[nz]) / R[nz]) < 1e-9


@pytest.mark.parametrize("kmin_q", [None, 0.3, 1.0])
def test_kdist_vs_oracle(small, kmin_q):
    ctx = small["ctx"]
    T, P = 1500.0, 0.1
    Kref, _, _ = oracle_state(small, T, P)
    kmin = 0.0 if kmin_q is None else float(np.quantile(Kref, kmin_q))
    if kmin_q is not None:
        Kref = np.maximum(Kref, kmin)
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0, kmin)
    r = ctx.kdist(Kref[None, :], nC=20, sorted_K=True, recon=True)
    nx = len(Kref)
    key, idx = oracle.bin_keys(NUMIN, NUMAX, DNU, nx, NBINS)
    Ks = oracle.sort_bins(Kref, idx, NBINS)
    assert np.array_equal(r["sorted"][0], Ks)
    co, nxmin, rec = oracle.kdist(Ks, nx // NBINS, NBINS, 20, kmin=kmin, recon=True)
    assert np.array_equal(r["nxmin"][0], nxmin)
    ok = nxmin < nx // NBINS          # empty bins print "0.0" coefficients
    if ok.any():
        assert np.max(np.abs(r["coeff"][0][ok] - co[ok])) < 1e-9


def test_end_to_end_coefficients_mixed(small):
    ctx = small["ctx"]
    T, P = 1500.0, 0.1
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    Km = ctx.opacity([T], [P], hkb.MIXED)
    r = ctx.kdist(Km, nC=20)
    Kref, _, _ = oracle_state(small, T, P)
    key, idx = oracle.bin_keys(NUMIN, NUMAX, DNU, len(Kref), NBINS)
    co, nxmin, _ = oracle.kdist(oracle.sort_bins(Kref, idx, NBINS), len(Kref) // NBINS,
                                NBINS, 20)
    err = np.max(np.abs(r["coeff"][0] - co))
    print(f"end-to-end Chebyshev max abs err (mixed): {err:.3e}")
    assert err < 1e-6


def test_errors_are_reported(small):
    ctx = small["ctx"]
    with pytest.raises(hkb.HkError) as e:
        ctx.set_grid(0.0, 1000.0, 0.3, 7)
    assert e.value.status == -4 and "evenly" in str(e.value)
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    with pytest.raises(hkb.HkError) as e:
        ctx.opacity([6000.0], [1.0])          # beyond the 1..5000 K q-table
    assert e.value.status == -4
    with pytest.raises(hkb.HkError) as e:
        ctx.opacity([1000.0], [1.0], precision=7)
    assert e.value.status == -1
    with hkb.Context(0) as c2:
        with pytest.raises(hkb.HkError) as e:
            c2.set_species(hkb.HITRAN, [18.0], [1.0])
            c2.opacity([1000.0], [1.0])
        assert e.value.status == -6


def test_table_graph_equals_opacity_and_kdist(small):
    """hk_table_build/hk_table_run (one CUDA graph for the whole T-P table;
    table mode 1: one persistent launch for the line prep and sums of every
    state) give the same bits as hk_opacity + hk_kdist on the same states, on
    every replay, and as the default per-batch graph."""
    import torch
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    Ts = np.array([300.0, 1000.0, 2500.0, 700.0, 1500.0, 120.0])
    Ps = np.array([1e-6, 1.0, 100.0, 1e-3, 0.1, 10.0])
    ns, nx, nC = len(Ts), ctx.nx, 20
    dev = torch.device("cuda")
    K = torch.empty((ns, nx), dtype=torch.float64, device=dev)
    coeff = torch.empty((ns, NBINS, nC), dtype=torch.float64, device=dev)
    nxmin = torch.empty((ns, NBINS), dtype=torch.int32, device=dev)
    ctx.set_table_mode(1)
    ctx.table_build(Ts, Ps, K, coeff, nxmin, nC=nC)
    ctx.set_table_mode(0)
    assert ctx.table_kernels == 2   # one persistent table launch + one fit launch
    ctx.table_run()
    ctx.table_status()
    K1, c1, n1 = K.cpu().numpy(), coeff.cpu().numpy(), nxmin.cpu().numpy()
    K.zero_()
    coeff.zero_()
    ctx.table_run()
    ctx.table_status()
    assert np.array_equal(K.cpu().numpy(), K1)
    assert np.array_equal(coeff.cpu().numpy(), c1)
    ctx.table_free()
    Kr = ctx.opacity(Ts, Ps, hkb.MIXED)
    fit = ctx.kdist(Kr, nC=nC)
    assert ctx.last_launches >= 4
    assert np.array_equal(K1, Kr)
    assert np.array_equal(c1, fit["coeff"])
    assert np.array_equal(n1, fit["nxmin"])
    # the default per-batch table graph gives the same bits
    ctx.table_build(Ts, Ps, K, coeff, nxmin, nC=nC)
    assert ctx.table_kernels == 4   # line prep, state scale, Voigt sum (one batch), fit
    ctx.table_run()
    ctx.table_status()
    assert np.array_equal(K.cpu().numpy(), K1)
    assert np.array_equal(coeff.cpu().numpy(), c1)
    ctx.table_free()


def test_small_table_graph_equals_opacity(small):
    """Tables of fewer than 4 states record the per-batch launches (line
    prep, state scale, Voigt sum, then the fit): same bits as hk_opacity +
    hk_kdist."""
    import torch
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    Ts, Ps = np.array([1500.0, 300.0]), np.array([0.1, 1e-3])
    ns, nx, nC = len(Ts), ctx.nx, 20
    dev = torch.device("cuda")
    K = torch.empty((ns, nx), dtype=torch.float64, device=dev)
    coeff = torch.empty((ns, NBINS, nC), dtype=torch.float64, device=dev)
    nxmin = torch.empty((ns, NBINS), dtype=torch.int32, device=dev)
    ctx.table_build(Ts, Ps, K, coeff, nxmin, nC=nC)
    assert ctx.table_kernels == 4
    ctx.table_run()
    ctx.table_status()
    K1, c1 = K.cpu().numpy(), coeff.cpu().numpy()
    ctx.table_free()
    Kr = ctx.opacity(Ts, Ps, hkb.MIXED)
    fit = ctx.kdist(Kr, nC=nC)
    assert np.array_equal(K1, Kr)
    assert np.array_equal(c1, fit["coeff"])


def test_sectioned_states_equal_batched(small):
    """A workspace too small for one state's line records runs each state in
    grid sections (the path of 5e8-line lists); K is bit-identical."""
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    Ts = np.array([1500.0, 300.0])
    Ps = np.array([0.1, 10.0])
    ref = {pr: ctx.opacity(Ts, Ps, pr) for pr in (hkb.MIXED, hkb.PLAIN_FP64)}
    assert ctx.count_pairs(1500.0, 0.1) == tuple(
        int(v) for v in (lambda w: ((w[:, 1] - w[:, 0]).sum() + (w[:, 5] - w[:, 4]).sum(),
                                    (w[:, 2] - w[:, 1]).sum() + (w[:, 4] - w[:, 3]).sum(),
                                    (w[:, 3] - w[:, 2]).sum()))(ctx.state_lines(1500.0, 0.1)[4]))
    try:
        ctx.set_workspace(prep_bytes=3000 * 112, part_bytes=4 * 2**30)
        for pr in (hkb.MIXED, hkb.PLAIN_FP64):
            K = ctx.opacity(Ts, Ps, pr)
            assert np.array_equal(K, ref[pr])
        assert ctx.last_launches > 6  # state pass + several sections per state
    finally:
        ctx.set_workspace()
