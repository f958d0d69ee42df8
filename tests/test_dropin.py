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
