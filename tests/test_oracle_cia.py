"""CPU: the oracle's restatement of readCiaFile (host.h:670-785) on
synthetic HITRAN-format CIA files, against the rules it follows.

Known answers: inside a set's nu range the value is the linear
interpolation of its table times rho NA / mass1 (rho = P 273.15 / T
amagat), plus kmin; a temperature equal to a set's takes that set; between
two sets the blend is linear in T; below the first set and above the last,
K = kmin; a set's last interval is reached only by the first grid point in
it (the reference's exit where nu reaches the header's numax)."""
import os

import numpy as np
import pytest

import oracle
from hkb import synth

MASS1 = 1.00794
NU = np.arange(100.0, 2000.1, 5.0)


def _file(tmp_path):
    f = str(tmp_path / "H2-H_2011.cia")
    sets = [(300.0, NU, 1e-46 * (1 + NU / 1000)), (500.0, NU, 3e-46 * (1 + NU / 1000)),
            (800.0, NU, 5e-46 * np.ones(len(NU))), (1200.0, NU[::4], 7e-46 * np.ones(len(NU[::4])))]
    synth.write_cia(f, sets, formula="H2-H")
    return f


def scale(T, P):
    return (P * 273.15 / T * oracle.AMAGAT) * (oracle.NA / MASS1)


def test_cia_rules(tmp_path):
    f = _file(tmp_path)
    x = oracle.grid_x(0.0, 0.5, 6000)
    inside = (x >= 100.0) & (x < 1995.0)
    for T, P in ((300.0, 1.0), (500.0, 2.0)):
        K = oracle.cia_opacity(f, 4, MASS1, x, T, P, kmin=1e-7)
        a = 1e-46 if T == 300.0 else 3e-46
        np.testing.assert_allclose(K[inside], a * (1 + x[inside] / 1000) * scale(T, P) + 1e-7, rtol=1e-12)
        assert np.all(K[x < 100.0] == 1e-7)
    # between 500 K and 800 K: linear in T
    K = oracle.cia_opacity(f, 4, MASS1, x, 650.0, 1.0, kmin=0.0)
    want = 0.5 * (3e-46 * (1 + x / 1000) + 5e-46) * scale(650.0, 1.0)
    np.testing.assert_allclose(K[inside], want[inside], rtol=1e-12)
    # below the first set and above the last: kmin
    assert np.all(oracle.cia_opacity(f, 4, MASS1, x, 250.0, 1.0, kmin=3.0) == 3.0)
    assert np.all(oracle.cia_opacity(f, 4, MASS1, x, 1300.0, 1.0, kmin=3.0) == 3.0)


def test_cia_last_interval(tmp_path):
    f = _file(tmp_path)
    x = oracle.grid_x(0.0, 0.5, 6000)
    K = oracle.cia_opacity(f, 4, MASS1, x, 300.0, 1.0)
    last = (x >= 1995.0) & (x < 2000.0)
    # only the first grid point of [1995, 2000) is evaluated
    assert K[last][0] > 0.0 and np.all(K[last][1:] == 0.0)
