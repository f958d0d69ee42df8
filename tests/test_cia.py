"""GPU: collision-induced absorption (hk_load_cia, param.dat ciaSystem)
against the oracle's restatement of readCiaFile (host.h:670-785).

The kernel applies the reference's rounded operations in the same order
(interpolation in nu, blend in T, rho and NA / mass1 scaling, kmin), so K is
compared bit for bit; the drop-in's text K (%.20g) too."""
import os
import sys

import numpy as np
import pytest

import hkb
import oracle
from hkb import synth

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import ref_run  # noqa: E402

pytestmark = pytest.mark.gpu

NU = np.arange(100.0, 2000.1, 5.0)
NUMIN, NUMAX, DNU, NBINS = 0.0, 3000.0, 0.5, 10


def _file(d):
    sets = [(300.0, NU, 1e-46 * (1 + NU / 1000)), (500.0, NU, 3e-46 * (1 + NU / 1000)),
            (800.0, NU[::3], 5e-46 * (2 - NU[::3] / 2000)), (1200.0, NU[::4], 7e-46 * np.ones(len(NU[::4])))]
    synth.write_cia(os.path.join(d, "H2-H_2011.cia"), sets, formula="H2-H")


def test_cia_matches_oracle(tmp_path):
    d = str(tmp_path) + "/"
    _file(d)
    with hkb.Context(0) as c:
        m1 = c.load_cia(d, "H2-H")
        assert m1 == 1.00794
        c.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0, kmin=2e-9)
        states = [(250.0, 1.0), (300.0, 1.0), (420.0, 0.3), (500.0, 2.0), (800.0, 1.0), (1000.0, 5.0),
                  (1300.0, 1.0)]
        T = np.array([s[0] for s in states])
        P = np.array([s[1] for s in states])
        K = c.opacity(T, P)
        x = oracle.grid_x(NUMIN, DNU, c.nx)
        for q, (Tq, Pq) in enumerate(states):
            want = oracle.cia_opacity(os.path.join(d, "H2-H_2011.cia"), 4, m1, x, Tq, Pq, kmin=2e-9)
            assert np.array_equal(K[q], want), (Tq, Pq, np.max(np.abs(K[q] - want)))
        # the k-distribution chain runs on it as on line opacities
        fit = c.kdist(K[1:2], nC=10)
        assert np.isfinite(fit["coeff"]).all()
    with hkb.Context(0) as c:
        with pytest.raises(hkb.HkError) as e:
            c.load_cia(d, "H2-H2")  # its 113 sets are not there
        assert e.value.status in (-2, -3)
        with pytest.raises(hkb.HkError) as e:
            c.load_cia(d, "CO-CO")
        assert e.value.status == -1


def test_dropin_cia(tmp_path):
    assert os.path.exists(ref_run.OUR_EXE), "build helios-k_b200/bin/heliosk first"
    d = str(tmp_path / "run")
    os.makedirs(d)
    _file(d + "/")
    ref_run.write_run(d, d, 650.0, 1.5, NUMIN, NUMAX, DNU, 25.0, NBINS, 10, store_k=1, resample=1,
                      ciaSystem="H2-H")
    r = ref_run.run(ref_run.OUR_EXE, d, timeout=300)
    assert r["rc"] == 0, r["tail"]
    out = np.loadtxt(os.path.join(d, "Out_syn.dat"))
    x = oracle.grid_x(NUMIN, DNU, len(out))
    want = oracle.cia_opacity(os.path.join(d, "H2-H_2011.cia"), 4, 1.00794, x, 650.0, 1.5)
    np.testing.assert_allclose(out[:, 1], want, rtol=1e-15, atol=0)
    assert os.path.exists(os.path.join(d, "Out_syn_cbin.dat"))
