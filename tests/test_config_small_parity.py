"""GPU parity on the small plain-method workload at its full size: 1e5
synthetic lines of one species (seed 0; nu0 ~ U[0, 30000], log10 S ~
U[-30, -18], E'' ~ Exp(3000), gamma_air ~ U[0.01, 0.1], n ~ U[0.4, 0.8]),
T = 1000 K, P = 1 atm, grid 0-30000 cm^-1 at 0.01 (3e6 points), cut
100 cm^-1, 300 bins of 10000 points, nC = 20.

The whole grid is summed on the GPU in both forms; the FP64 oracle sums 16
whole bins drawn at random (about 1e7 pairs each), which are compared point
by point, and their per-bin sort and Chebyshev fit are compared with the
oracle's fit of the oracle's K.

Tolerances (written here): K 1e-5 (mixed) and 1e-12 (plain FP64) relative
where K > 1e-6 of its bin maximum; the mixed form's Chebyshev coefficients
1e-6 absolute, the plain form's 1e-9; Nxmin equal.
"""
import numpy as np
import pytest

import hkb
import oracle
from hkb import synth

pytestmark = pytest.mark.gpu

W = synth.WORKLOADS["small"]
NBINS_CHECKED = 16


def test_small_workload_full_size():
    L = synth.hitran_lines(W["n"], seed=W["seed"], logS=W["logS"])
    Tq, Qq = synth.q_table()
    T, P = W["T"][0], W["P"][0]
    nbins, nC = W["nbins"], W["nC"]
    with hkb.Context(0) as ctx:
        ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
        ctx.set_partition(0, Tq, Qq)
        ctx.set_options(qalphaL=1.0)
        ctx.load_lines_hitran(L)
        ctx.set_grid(W["numin"], W["numax"], W["dnu"], nbins, 0, W["cut"])
        nx = ctx.nx
        assert nx == 3_000_000
        K = {pr: ctx.opacity([T], [P], pr)[0] for pr in (hkb.MIXED, hkb.PLAIN_FP64)}
        fit = {pr: ctx.kdist(K[pr][None, :], nC=nC) for pr in K}
    nxb = nx // nbins
    Q = oracle.partition(Tq, Qq, T)
    nu, S, iad, vy = oracle.prep_hitran(L, [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    win = oracle.windows(nu, S, iad, vy, W["numin"], W["dnu"], nx, 0, W["cut"])
    bins = np.sort(np.random.default_rng(0).choice(nbins, NBINS_CHECKED, replace=False))
    worst = {pr: 0.0 for pr in K}
    cworst = {pr: 0.0 for pr in K}
    npts = 0
    for b in bins:
        ib, ie = int(b) * nxb, (int(b) + 1) * nxb
        Kref, _ = oracle.opacity(nu, S, iad, vy, win, W["numin"], W["dnu"], nx, irange=(ib, ie))
        mask = Kref > 1e-6 * Kref.max()
        npts += int(mask.sum())
        co, nxmin, _ = oracle.kdist(np.sort(Kref), nxb, 1, nC)
        for pr in K:
            Kg = K[pr][ib:ie]
            worst[pr] = max(worst[pr], float(np.max(np.abs(Kg[mask] - Kref[mask]) / Kref[mask])))
            assert fit[pr]["nxmin"][0, b] == nxmin[0]
            cworst[pr] = max(cworst[pr], float(np.max(np.abs(fit[pr]["coeff"][0, b] - co[0]))))
    print(f"small workload, {NBINS_CHECKED} bins ({npts} points): K max rel err mixed "
          f"{worst[hkb.MIXED]:.2e} plain {worst[hkb.PLAIN_FP64]:.2e}; Chebyshev max abs err "
          f"mixed {cworst[hkb.MIXED]:.2e} plain {cworst[hkb.PLAIN_FP64]:.2e}")
    assert worst[hkb.MIXED] < 1e-5
    assert worst[hkb.PLAIN_FP64] < 1e-12
    assert cworst[hkb.MIXED] < 1e-6
    assert cworst[hkb.PLAIN_FP64] < 1e-9
