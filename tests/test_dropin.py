"""GPU: the drop-in executable (helios-k_b200/bin/heliosk) run like the
reference -- param.dat, <species>.param, partition file, binary line file in,
Info/Out files out -- against the FP64 oracle.

Tolerances (written here): grid wavenumbers bit-exact; K 1e-5 relative where
K > 1e-6 of its bin maximum; Chebyshev coefficients 1e-6 absolute.
"""
import os
import sys

import numpy as np
import pytest

import oracle
from hkb import synth

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import ref_run  # noqa: E402

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS, NC, CUT = 1000.0, 1300.0, 0.01, 10, 20, 25.0


def test_dropin_outputs_match_oracle(tmp_path):
    assert os.path.exists(ref_run.OUR_EXE), "build helios-k_b200/bin/heliosk first"
    L = synth.hitran_lines(3000, seed=17, nu_min=NUMIN - 40.0, nu_max=NUMAX + 40.0)
    T, P = 900.0, 0.5
    d = str(tmp_path / "run")
    ref_run.make_run_dir(d, L, T, P, NUMIN, NUMAX, DNU, CUT, NBINS, NC, store_k=1, resample=1)
    r = ref_run.run(ref_run.OUR_EXE, d, timeout=300)
    assert r["rc"] == 0, r["tail"]
    assert "K(x)" in r["info"] and "Lines" in r["info"]
    out = np.loadtxt(os.path.join(d, "Out_syn.dat"))
    x, K = out[:, 0], out[:, 1]
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    assert np.array_equal(x, oracle.grid_x(NUMIN, DNU, nx))
    # the file's lines were read back from the binary records (float64 fields)
    Lr = synth.read_hitran_bin(os.path.join(d, "syn.bin"))
    Tq, Qq = synth.q_table()
    Q = oracle.partition(Tq, Qq, T)
    nu, S, iad, vy = oracle.prep_hitran(Lr, [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, CUT)
    Kref, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx)
    Kb, Rb = K.reshape(NBINS, -1), Kref.reshape(NBINS, -1)
    m = Rb > 1e-6 * Rb.max(axis=1, keepdims=True)
    err = np.max(np.abs(Kb - Rb)[m] / Rb[m])
    print(f"drop-in K max rel err {err:.2e}; times {r['info']}")
    assert err < 1e-5
    key, idx = oracle.bin_keys(NUMIN, NUMAX, DNU, nx, NBINS)
    co, nxmin, _ = oracle.kdist(oracle.sort_bins(Kref, idx, NBINS), nx // NBINS, NBINS, NC)
    cb = ref_run.read_cbin(d)
    assert cb.shape == (NBINS, NC + 2)
    assert np.allclose(cb[:, 1], np.minimum(nxmin / (nx // NBINS - 1), 1.0), rtol=0, atol=1e-15)
    ce = np.max(np.abs(cb[:, 2:] - co.reshape(NBINS, NC)))
    print(f"drop-in Chebyshev max abs err {ce:.2e}")
    assert ce < 1e-6


def test_dropin_means_and_transmission(tmp_path):
    """doMean = 1 and doTransmission = 1 (heliosk.cu:1953-2020, 2377-2430):
    Out_<name>_mean.dat and Out_<name>_tr.dat against the oracle chain
    (opacity, per-bin sort, fit and reconstruction, means, transmission).
    Tolerance 1e-5 relative (the mixed-form K's error bound)."""
    assert os.path.exists(ref_run.OUR_EXE), "build helios-k_b200/bin/heliosk first"
    L = synth.hitran_lines(3000, seed=17, nu_min=NUMIN - 40.0, nu_max=NUMAX + 40.0)
    T, P = 900.0, 0.5
    # K here (internal units) spans 2e11 .. 1e30: m = e^-75 .. e^73.5 takes
    # Tr from 1 down to 0 (10 % of the values lie in (0.01, 0.99))
    nTr, dTr = 100, 1.5
    d = str(tmp_path / "run")
    ref_run.make_run_dir(d, L, T, P, NUMIN, NUMAX, DNU, CUT, NBINS, NC, store_k=0, resample=1,
                         doMean=1, doTransmission=1, nTr=nTr, dTr=dTr)
    r = ref_run.run(ref_run.OUR_EXE, d, timeout=300)
    assert r["rc"] == 0, r["tail"]
    assert "mean K(x)" in r["info"] and "Transmission" in r["info"]
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    x = oracle.grid_x(NUMIN, DNU, nx)
    Lr = synth.read_hitran_bin(os.path.join(d, "syn.bin"))
    Tq, Qq = synth.q_table()
    Q = oracle.partition(Tq, Qq, T)
    nu, S, iad, vy = oracle.prep_hitran(Lr, [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, CUT)
    Kref, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx)
    # means: Planck, Rosseland, sum B dnu, analytic, sum dB/dT dnu, analytic
    mean = np.loadtxt(os.path.join(d, "Out_syn_mean.dat"))
    m = oracle.means(x, Kref, T)
    want = [m[0] / m[2], m[3] / m[1], m[2] * DNU, None, m[3] * DNU, None]
    for k, w in enumerate(want):
        if w is not None:
            assert mean[k] == pytest.approx(w, rel=1e-5), k
    # the analytic integrals (the grid covers part of the spectrum, so the
    # numeric ones are smaller)
    kb, h, c = 1.3806489e-16, 6.62606957e-27, 2.99792458e10
    sigma = 2.0 * kb**4 / (h**3 * c**2 * 15.0) * np.pi**5
    assert mean[3] == pytest.approx(sigma * T**4 / np.pi, rel=1e-12)
    assert mean[5] == pytest.approx(4.0 * sigma * T**3 / np.pi, rel=1e-12)
    assert mean[2] < mean[3] and mean[4] < mean[5]
    # transmission of the reconstructed bins
    nxb = nx // NBINS
    key, idx = oracle.bin_keys(NUMIN, NUMAX, DNU, nx, NBINS)
    Ks = oracle.sort_bins(Kref, idx, NBINS)
    co, nxmin, rec = oracle.kdist(Ks, nxb, NBINS, NC, recon=True)
    Tr_ref = oracle.transmission(rec, nxb, NBINS, nxmin, 0.0, nTr, dTr)
    tr = np.loadtxt(os.path.join(d, "Out_syn_tr.dat"))
    assert tr.shape == (NBINS * nTr, 2)
    mm = np.exp((np.arange(nTr) - nTr // 2) * dTr)
    np.testing.assert_allclose(tr[:, 0], np.tile(mm, NBINS), rtol=1e-15)
    # Tr lies in [0, 1]; where exp(-K m) underflows both are ~0 (atol)
    big = Tr_ref.ravel() > 1e-12
    assert big.sum() > NBINS * nTr // 5 and Tr_ref.max() > 0.9
    err = np.max(np.abs(tr[big, 1] - Tr_ref.ravel()[big]) / Tr_ref.ravel()[big])
    print(f"drop-in means {mean[:2]}, transmission max rel err {err:.2e} (Tr > 1e-12)")
    np.testing.assert_allclose(tr[:, 1], Tr_ref.ravel(), rtol=1e-5, atol=1e-12)


def test_dropin_mixture_profile_sublorentzian(tmp_path):
    """SpeciesFile (two species), profile = 2 with removePlinth = 1 and a
    subLorentzianfile in the reference's layouts (host.h:463-515): the
    drop-in's K against the oracle chain, 1e-9 relative (plinth removal runs
    the FP64 form)."""
    assert os.path.exists(ref_run.OUR_EXE), "build helios-k_b200/bin/heliosk first"
    d = str(tmp_path / "run")
    os.makedirs(d)
    T, P = 900.0, 0.5
    specs = {"spa": ("11", 18.0106, 41), "spb": ("26", 28.0101, 42)}
    ab = {"spa": 2e-3, "spb": 5e-4}
    lines = {}
    for name, (cid, m, seed) in specs.items():
        L = synth.hitran_lines(4000, seed=seed, nu_min=NUMIN - 40.0, nu_max=NUMAX + 40.0)
        synth.write_species(d, name, database=0, nfiles=1, nl=[4000],
                            limits=(int(NUMIN - 50), int(NUMAX + 50)), isos=[(cid, 1.0, m)])
        synth.write_hitran_bin(os.path.join(d, name + ".bin"), L, cids=np.array([(" " + cid).encode()] * 4000))
        lines[name] = L
    with open(os.path.join(d, "species.dat"), "w") as f:
        for name in specs:
            f.write(f"{name} {ab[name]}\n")
    sl14 = [3.0, 10.0, 20.0, 0.09, -0.05, 0.004, 0.05, 0.02, 0.003, 0.02, 0.0, 0.0, 1050.0, 1250.0]
    with open(os.path.join(d, "sl.dat"), "w") as f:
        f.write(f"sigma1 {sl14[0]}\nsigma2 {sl14[1]}\nsigma3 {sl14[2]}\nB alpha beta epsilon\n")
        for k in range(3):
            f.write(f"B{k + 1} {sl14[3 + 3 * k]} {sl14[4 + 3 * k]} {sl14[5 + 3 * k]}\n")
        f.write(f"range lo hi\n{sl14[12]} {sl14[13]}\n")
    ref_run.write_run(d, d, T, P, NUMIN, NUMAX, DNU, CUT, NBINS, NC, store_k=1, resample=0,
                      SpeciesFile=os.path.join(d, "species.dat"), profile=2, removePlinth=1,
                      subLorentzianfile=os.path.join(d, "sl.dat"))
    r = ref_run.run(ref_run.OUR_EXE, d, timeout=300)
    assert r["rc"] == 0, r["tail"]
    K = np.loadtxt(os.path.join(d, "Out_syn.dat"))[:, 1]
    Tq, Qq = synth.q_table()
    Q = oracle.partition(Tq, Qq, T)
    mean_mass = sum(ab[n] * specs[n][1] for n in specs)
    cols = [oracle.prep_hitran(lines[n], [specs[n][1]], [1.0], [Q], T, P, qalphaL=1.0, units=0,
                               meanMass=mean_mass, Sscale=ab[n]) for n in specs]
    nu, S, iad, vy = (np.concatenate([c[k] for c in cols]) for k in range(4))
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, CUT, profile=2)
    pl = oracle.plinth(S, iad, vy, win, 0, CUT, 2)
    Kref, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx, profile=2, plinth=pl,
                             sublorentz=oracle.sublorentz_params(sl14, T))
    # the drop-in writes K * unitScale (units 0: 1) as %.20g
    Rb, Kb = Kref.reshape(NBINS, -1), K.reshape(NBINS, -1)
    m = Rb > 1e-6 * Rb.max(axis=1, keepdims=True)
    err = np.max(np.abs(Kb - Rb)[m] / Rb[m])
    print(f"drop-in mixture + Lorentz + plinth + sub-Lorentzian: max rel err {err:.2e}")
    assert err < 1e-9
