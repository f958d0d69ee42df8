"""GPU: species mixtures (hk_load_mixture, param.dat SpeciesFile) against the
FP64 oracle restating the reference's per-species loop (heliosk.cu:660-700,
784-800): each species' strengths scaled by its abundance, the mean molar
mass (units 0) taken over the whole mixture, all species summed into one K.

Tolerances (written here): mixed form 1e-5, plain FP64 1e-12 relative where
K > 1e-6 of its bin maximum; a one-species mixture is bit-identical to
hk_load_species_file (the abundance is ignored, as the reference does).
"""
import os

import numpy as np
import pytest

import hkb
import oracle
from hkb import synth
from test_gpu_parity import masked_relerr

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS, CUT = 1000.0, 1600.0, 0.01, 20, 25.0
SPECIES = {
    "spa": dict(isos=[("11", 0.99, 18.0106), ("12", 0.01, 20.0148)], n=40000, seed=3),
    "spb": dict(isos=[("26", 0.987, 28.0101)], n=25000, seed=4),
}
ABUND = {"spa": 3.0e-3, "spb": 7.0e-4}


def _write(d):
    lines = {}
    for name, sp in SPECIES.items():
        L = synth.hitran_lines(sp["n"], seed=sp["seed"], nu_min=NUMIN - 30.0, nu_max=NUMAX + 30.0)
        rng = np.random.default_rng(sp["seed"] + 100)
        L["iso"] = rng.integers(0, len(sp["isos"]), sp["n"]).astype(np.int32)
        L["gself"] = rng.uniform(0.05, 0.3, sp["n"])
        synth.write_species(d, name, database=0, nfiles=1, nl=[sp["n"]],
                            limits=(int(NUMIN - 40), int(NUMAX + 40)), isos=sp["isos"])
        cid = np.array([(" %s" % c).encode() for c, _, _ in sp["isos"]])
        synth.write_hitran_bin(os.path.join(d, name + ".bin"), L, cids=cid[L["iso"]])
        lines[name] = L
    return lines


def _oracle(lines, names, T, P, qalphaL, units):
    Tq, Qq = synth.q_table()
    Q = oracle.partition(Tq, Qq, T)
    ab = [ABUND[n] if len(names) > 1 else 1.0 for n in names]
    mean_mass = sum(a * sum(i[1] * i[2] for i in SPECIES[n]["isos"]) for n, a in zip(names, ab))
    cols = []
    for n, a in zip(names, ab):
        iso = SPECIES[n]["isos"]
        cols.append(oracle.prep_hitran(lines[n], [i[2] for i in iso], [i[1] for i in iso],
                                       [Q] * len(iso), T, P, qalphaL=qalphaL, units=units,
                                       meanMass=mean_mass, Sscale=a))
    nu, S, iad, vy = (np.concatenate([c[k] for c in cols]) for k in range(4))
    nx = oracle.grid_nx(NUMIN, NUMAX, DNU)
    win = oracle.windows(nu, S, iad, vy, NUMIN, DNU, nx, 0, CUT)
    K, _ = oracle.opacity(nu, S, iad, vy, win, NUMIN, DNU, nx)
    return K


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("mix")) + "/"
    return d, _write(d)


@pytest.mark.parametrize("units", [0, 1])
def test_mixture_matches_oracle(files, units):
    d, lines = files
    names = ["spa", "spb"]
    with hkb.Context(0) as c:
        c.set_options(qalphaL=0.6, units=units)
        c.load_mixture(d, names, [ABUND[n] for n in names], NUMIN, NUMAX, 0, CUT)
        assert c.num_lines == sum(SPECIES[n]["n"] for n in names)
        c.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, CUT)
        for T, P in ((1200.0, 0.3), (400.0, 5.0)):
            Kref = _oracle(lines, names, T, P, 0.6, units)
            for prec, tol in ((hkb.MIXED, 1e-5), (hkb.PLAIN_FP64, 1e-12)):
                K = c.opacity([T], [P], prec)[0]
                err, _ = masked_relerr(K, Kref, NBINS)
                print(f"units {units} T={T} P={P} prec {prec} err {err:.2e}")
                assert err < tol


def test_one_species_mixture_equals_species_file(files):
    d, _ = files
    with hkb.Context(0) as a, hkb.Context(0) as b:
        a.load_species_file(d, "spa", NUMIN, NUMAX, 0, CUT)
        b.load_mixture(d, ["spa"], [0.25], NUMIN, NUMAX, 0, CUT)  # abundance ignored for one
        for c in (a, b):
            c.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, CUT)
        assert np.array_equal(a.opacity([900.0], [1.0]), b.opacity([900.0], [1.0]))


def test_mixture_errors(files):
    d, _ = files
    synth.write_species(d, "exo", database=2, nfiles=1, nl=[10], limits=(1000, 1600),
                        defaultL=0.07, defaultn=0.5)
    synth.write_exomol_bin(os.path.join(d, "exo.bin"), synth.exomol_lines(10, nu_max=1500.0))
    with hkb.Context(0) as c:
        with pytest.raises(hkb.HkError) as e:
            c.load_mixture(d, ["spa", "exo"], [1.0, 1.0], NUMIN, NUMAX, 0, CUT)
        assert e.value.status == -8
        with pytest.raises(hkb.HkError) as e:
            c.load_mixture(d, ["spa", "nothere"], [1.0, 1.0], NUMIN, NUMAX, 0, CUT)
        assert e.value.status == -2
        with pytest.raises(hkb.HkError) as e:
            c.load_mixture(d, ["spa", "spb"], [1.0, -1.0], NUMIN, NUMAX, 0, CUT)
        assert e.value.status == -1
