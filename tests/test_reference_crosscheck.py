"""GPU: the FP64 oracle's Voigt sum cross-checked against the reference's own
CUDA program (HELIOS-K heliosk.cu compiled unmodified for sm_100a into
oracle/_ref/ by `make -C oracle ref`) on one synthetic run directory.

The reference ships no line list, so its Voigt sum has no golden vector;
this run is the only reference-side pin of the sum (Line6A/B/C_Call and the
Line6f kernels, voigt.h:1177-2036).  The reference evaluates the line-centre
offset in FP32 (its error is 0.015-0.022 Doppler widths at these
wavenumbers) and writes K as float32 (Out_<name>.bin, doStoreFullK = 2), so
the comparison is loose by design; strengths stay in log10 S in [-40, -36],
where the reference's FP32 strengths neither overflow nor flush.

Bounds (written here), where K > 1e-6 of its bin maximum: median relative
difference below 1e-4, maximum below 5e-2; the reference's Chebyshev
coefficients (Out_<name>_cbin.dat) within 5e-2 absolute of the oracle's fit
of the oracle's K, median within 1e-3.  The same inputs through this
library's drop-in executable are held to the library's own bound, 1e-5.
"""
import os
import sys

import numpy as np
import pytest

import oracle
from hkb import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_run  # noqa: E402

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS, NC, CUT = 1000.0, 1300.0, 0.01, 10, 20, 25.0
T, P = 900.0, 0.5


def _rel(K, Kref):
    Kb, Rb = K.reshape(NBINS, -1), Kref.reshape(NBINS, -1)
    m = Rb > 1e-6 * Rb.max(axis=1, keepdims=True)
    return np.abs(Kb - Rb)[m] / Rb[m]


@pytest.mark.skipif(not os.path.exists(ref_run.REF_EXE),
                    reason="oracle/_ref/heliosk absent (make -C oracle ref needs the reference sources)")
def test_oracle_sum_against_reference_build(tmp_path):
    L = synth.hitran_lines(3000, seed=23, logS=(-40.0, -36.0), nu_min=NUMIN - 40.0,
                           nu_max=NUMAX + 40.0)
    runs = {}
    for tag, exe in (("ref", ref_run.REF_EXE), ("ours", ref_run.OUR_EXE)):
        d = str(tmp_path / tag)
        ref_run.make_run_dir(d, L, T, P, NUMIN, NUMAX, DNU, CUT, NBINS, NC, store_k=2, resample=1)
        r = ref_run.run(exe, d, timeout=300)
        assert r["rc"] == 0, r["tail"]
        runs[tag] = (ref_run.read_k(d).astype(np.float64), ref_run.read_cbin(d))
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    Lr = synth.read_hitran_bin(str(tmp_path / "ref" / "syn.bin"))
    Tq, Qq = synth.q_table()
    Q = oracle.partition(Tq, Qq, T)
    nu, S, iad, vy = oracle.prep_hitran(Lr, [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, CUT)
    Kref, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx)
    key, idx = oracle.bin_keys(NUMIN, NUMAX, DNU, nx, NBINS)
    co, nxmin, _ = oracle.kdist(oracle.sort_bins(Kref, idx, NBINS), nx // NBINS, NBINS, NC)

    Kr, cb = runs["ref"]
    assert Kr.shape == (nx,) and cb.shape == (NBINS, NC + 2)
    e = _rel(Kr, Kref)
    ce = np.abs(cb[:, 2:] - co)
    print(f"reference build vs oracle: K rel diff median {np.median(e):.2e} "
          f"p99 {np.quantile(e, 0.99):.2e} max {e.max():.2e} over {e.size} points; "
          f"Chebyshev abs diff median {np.median(ce):.2e} max {ce.max():.2e}")
    assert np.median(e) < 1e-4 and e.max() < 5e-2
    assert np.median(ce) < 1e-3 and ce.max() < 5e-2

    Ko, cbo = runs["ours"]
    eo = _rel(Ko, Kref)
    # float32 output file: half an ulp of float32 on top of the library's 1e-5
    print(f"drop-in vs oracle: K rel diff max {eo.max():.2e}")
    assert eo.max() < 1e-5 + 6e-8
    assert np.max(np.abs(cbo[:, 2:] - co)) < 1e-6
