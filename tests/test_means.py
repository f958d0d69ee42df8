"""GPU: hk_means and hk_transmission (C ABI) against the FP64 oracle.

Tolerances (written here): the four mean sums 1e-12 relative (FP64 sums in
another order); the transmission function 1e-12 relative.  Inputs are this
library's own mixed-form opacities of the small workload (with a band set to
K = 0, which the Rosseland sum skips), sorted or reconstructed by hk_kdist
with Nxmin > 0 from a kmin inside the bins' range.
"""
import numpy as np
import pytest

import hkb
import oracle
from hkb import synth

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS = 0.0, 3000.0, 0.01, 30
STATES = [(1500.0, 0.1), (300.0, 1e-6), (2000.0, 100.0)]


@pytest.fixture(scope="module")
def small():
    L = synth.hitran_lines(20000, seed=11, nu_max=3000.0)
    Tq, Qq = synth.q_table()
    ctx = hkb.Context(0)
    ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
    ctx.set_partition(0, Tq, Qq)
    ctx.set_options(qalphaL=1.0)
    ctx.load_lines_hitran(L)
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    Ts = np.array([s[0] for s in STATES])
    Ps = np.array([s[1] for s in STATES])
    K = ctx.opacity(Ts, Ps, hkb.MIXED)
    yield dict(ctx=ctx, K=K, T=Ts, x=oracle.grid_x(NUMIN, DNU, ctx.nx))
    ctx.close()


def test_means_match_oracle(small):
    ctx, Ts = small["ctx"], small["T"]
    K = small["K"].copy()
    K[:, 5000:6000] = 0.0  # the Rosseland sum skips K = 0 points
    got = ctx.means(Ts, K)
    for s in range(len(Ts)):
        want = oracle.means(small["x"], K[s], Ts[s])
        np.testing.assert_allclose(got[s], want, rtol=1e-12, atol=0)
        print(f"T={Ts[s]} Planck {got[s, 0] / got[s, 2]:.6e} Rosseland {got[s, 3] / got[s, 1]:.6e}")
    # device input, same sums
    import torch
    Kd = torch.from_numpy(K).cuda()
    np.testing.assert_array_equal(ctx.means(Ts, Kd), got)


def test_transmission_sorted_and_fit(small):
    ctx, K = small["ctx"], small["K"]
    nxb = ctx.nx // NBINS
    nTr, dTr = 64, 2.0  # m = e^-64 .. e^62 reaches these states' K (1e-5 .. 1e50)
    fit = ctx.kdist(K, nC=20, sorted_K=True)
    Ks = fit["sorted"]
    got = ctx.transmission(Ks, None, nTr, dTr)
    for s in range(K.shape[0]):
        want = oracle.transmission(Ks[s], nxb, NBINS, None, 0.0, nTr, dTr)
        np.testing.assert_allclose(got[s], want, rtol=1e-12, atol=1e-290)
    # with the fit: kmin inside the bins' values gives Nxmin > 0
    kmin = float(np.median(K[0]))
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0, kmin=kmin)
    try:
        fr = ctx.kdist(K, nC=20, recon=True)
        assert (fr["nxmin"] > 0).any()
        got = ctx.transmission(fr["recon"], fr["nxmin"], nTr, dTr)
        for s in range(K.shape[0]):
            want = oracle.transmission(fr["recon"][s], nxb, NBINS, fr["nxmin"][s], kmin, nTr, dTr)
            np.testing.assert_allclose(got[s], want, rtol=1e-12, atol=1e-290)
        import torch
        gd = ctx.transmission(torch.from_numpy(fr["recon"]).cuda(),
                              torch.from_numpy(fr["nxmin"]).cuda(), nTr, dTr)
        np.testing.assert_array_equal(gd, got)
    finally:
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)


def test_errors(small):
    ctx, K = small["ctx"], small["K"]
    with pytest.raises(hkb.HkError) as e:
        ctx.means([0.0, 1.0, 2.0], K)
    assert e.value.status == -4
    with pytest.raises(hkb.HkError) as e:
        ctx.transmission(K, None, 0, 0.1)
    assert e.value.status == -4
