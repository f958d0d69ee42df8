"""Pin the FP64 oracle to the reference's own golden run (plots/p004).

plots/p004 is the one self-consistent k-distribution run the reference ships
(30000 points, 1 bin, nC = 20, kmin = 0); tests/golden/make_p004.py turns its
text outputs into tests/golden/p004.npz.
"""
import numpy as np
import pytest

import oracle

BIN1 = np.array([0, 30000, 30000], np.int32)


def test_p004_sort_is_bit_exact(golden_p004):
    # heliosk.cu:2046-2051 sort of Out_i.dat == Out_i_bin.dat, bit for bit
    s = oracle.sort_bins(golden_p004["K_i"], BIN1, 1)
    assert np.array_equal(s, golden_p004["Ksorted_i"])


def test_p004_chebyshev_fit(golden_p004):
    Ks = oracle.sort_bins(golden_p004["K_r"], BIN1, 1)
    coeff, nxmin, rec = oracle.kdist(Ks, 30000, 1, 20, kmin=0.0, recon=True)
    cb = golden_p004["cbin_r"]
    # Out_r_cbin.dat: kmin, ystart = min(Nxmin/(Nxb-1), 1), c0..c19
    assert cb[0] == 0.0
    assert nxmin[0] == 4533
    assert min(nxmin[0] / 29999.0, 1.0) == cb[1]
    assert np.max(np.abs(coeff[0] - cb[2:])) < 1e-10
    R = golden_p004["Krecon_r"]
    nz = R != 0
    assert np.array_equal(rec[~nz], R[~nz])
    assert np.max(np.abs(rec[nz] - R[nz]) / R[nz]) < 1e-10


def test_p004_full_least_squares_differs():
    """The reference applies nc-1 of the nc reflections (resample.h:251);
    a true least-squares fit gives visibly different coefficients, so the
    golden match above pins that quirk."""
    g = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__),
                                            "golden", "p004.npz"))
    Ks = oracle.sort_bins(g["K_r"], BIN1, 1)
    nx = 4533
    K2 = Ks.copy()
    # same rescale + ln as the reference, then a textbook least squares
    j = np.arange(30000)
    ii = nx + (1 - nx / 29999.0) * j
    ii = np.where(ii >= 29999, 0.999999 * 29999, ii)
    il = (ii / 30000.0 * 30000).astype(int)
    K2 = Ks[il] + (Ks[il + 1] - Ks[il]) * (ii - il)
    b = np.log(K2)
    t = j * 2.0 / 29999.0 - 1.0
    V = np.polynomial.chebyshev.chebvander(t, 19)
    c = np.linalg.lstsq(V, b, rcond=None)[0]
    assert np.max(np.abs(c - g["cbin_r"][2:])) > 1e-3


def test_partition_interpolation_rules():
    T = np.arange(1.0, 11.0)
    Q = 0.1 * T ** 1.5
    # exact table point: first row with T1 >= T is that row
    assert oracle.partition(T, Q, 5.0) == pytest.approx(Q[4], rel=1e-15)
    # linear interpolation between rows (host.h:57-59)
    v = oracle.partition(T, Q, 5.25)
    assert v == (Q[5] - Q[4]) * 0.25 + Q[4]
    # below the table: error (host.h:49-52); beyond the end: error (EOF)
    with pytest.raises(ValueError):
        oracle.partition(T, Q, 0.5)
    with pytest.raises(ValueError):
        oracle.partition(T, Q, 11.0)
    # duplicated temperature rows before T: error (host.h:45-48)
    with pytest.raises(ValueError):
        oracle.partition(np.array([1.0, 2.0, 2.0, 3.0]), np.ones(4), 2.5)


@pytest.mark.parametrize("numin,numax,dnu,nbins", [
    (0.0, 30000.0, 0.01, 300),     # small / hitemp / table grids
    (1000.0, 10000.0, 0.01, 300),  # adjoint grid
    (0.0, 40000.0, 0.01, 400),     # exomol grid
    (0.0, 30000.0, 1.0, 1),        # p004 grid
])
def test_bin_keys_are_equal_blocks(numin, numax, dnu, nbins):
    """binKey_kernel (voigt.h:779-805) on these grids puts point i in bin
    i // Nxb, the layout the fused sort+fit kernel assumes."""
    nx = oracle.grid_nx(numin, numax, dnu)
    assert nx % nbins == 0
    key, idx = oracle.bin_keys(numin, numax, dnu, nx, nbins)
    nxb = nx // nbins
    assert np.array_equal(key, np.arange(nx) // nxb)
    assert np.array_equal(idx[:nbins + 1], np.arange(nbins + 1) * nxb)


def test_find_cut_rules():
    nxb, nb = 10, 3
    K = np.concatenate([
        np.array([0, 0, 0, 1, 2, 3, 4, 5, 6, 7.0]),   # transition after 3 zeros
        np.zeros(10),                                  # empty bin
        np.array([0, 0, 0, 0, 0, 0, 0, 0, 0, 9.0]),   # last bin, id NL-3 rule
    ])
    nxmin = np.empty(nb, np.int32)
    lib = oracle.lib()
    lib.hko_find_cut(oracle._ptr(K), len(K), nxb, 0.0, nb, oracle._ptr(nxmin))
    # the last bin: K[NL-3] <= kmin sets Nxb, then the later transition at
    # id NL-2 (K[NL-2] <= kmin < K[NL-1]) wins
    assert list(nxmin) == [3, 10, 9]
    K[-2] = 8.0  # transition at NL-3 itself: the NL-3 rule overrides it
    lib.hko_find_cut(oracle._ptr(K), len(K), nxb, 0.0, nb, oracle._ptr(nxmin))
    assert list(nxmin) == [3, 10, 10]
