"""GPU: the streamed line-file loader (hk_load_species_file) against the
array loaders (hk_load_lines_hitran / _exomol) on the same records.

Both routes end in the same device columns, sorted by centre on the GPU, so
every per-line quantity of a state and the opacity must be bit-identical.
The files hold more records than one loader chunk (2^20), are split over
several files and isotopologues, and include the reference's error cases:
an isotopologue id missing from the species table (host.h:636-639) and a
file shorter than its declared line count.
"""
import os

import numpy as np
import pytest

import hkb
from hkb import synth

pytestmark = pytest.mark.gpu

ISOS = [("11", 0.997, 18.0106), ("12", 2.0e-3, 20.0148), ("13", 3.7e-4, 19.0148)]
NUMIN, NUMAX, DNU, NBINS, CUT = 1000.0, 1300.0, 0.01, 10, 25.0


def _two_iso_lines(n, seed):
    L = synth.hitran_lines(n, seed=seed, nu_min=0.0, nu_max=20000.0)
    rng = np.random.default_rng(seed + 1)
    L["iso"] = rng.choice(len(ISOS), size=n, p=[0.8, 0.15, 0.05]).astype(np.int32)
    # every column non-uniform, so each is gathered rather than kept as a scalar
    L["A"] = rng.uniform(0.0, 50.0, n)
    L["delta"] = rng.uniform(-0.01, 0.01, n)
    L["gself"] = rng.uniform(0.05, 0.4, n)
    return L


def _write_files(d, L, limits, species="syn2"):
    """Line files split at the wavenumber limits (the reference's
    <species>_<lo>-<hi>.bin names); records keep their file order."""
    nu = L["nu"]
    parts, nl = [], []
    for lo, hi in zip(limits[:-1], limits[1:]):
        m = (nu >= lo) & (nu < hi)
        parts.append(np.nonzero(m)[0])
        nl.append(int(m.sum()))
    synth.write_species(d, species, database=0, nfiles=len(nl), nl=nl, limits=limits, isos=ISOS)
    cid = np.array([(" %s" % c).encode() for c, _, _ in ISOS])
    for k, idx in enumerate(parts):
        name = "%s_%05d-%05d.bin" % (species, limits[k], limits[k + 1]) if len(nl) > 1 else species + ".bin"
        synth.write_hitran_bin(os.path.join(d, name), {k2: v[idx] for k2, v in L.items()},
                               cids=cid[L["iso"][idx]])
    return np.concatenate(parts)


def _ctx_arrays(L, order, qalphaL, gammaF):
    c = hkb.Context(0)
    c.set_options(qalphaL=qalphaL, gammaF=gammaF)
    c.set_species(hkb.HITRAN, [m for _, _, m in ISOS], [a for _, a, _ in ISOS])
    T, Q = synth.q_table()
    for j in range(len(ISOS)):
        c.set_partition(j, T, Q)
    c.load_lines_hitran({k: v[order] for k, v in L.items()})
    return c


def test_species_file_equals_arrays(tmp_path):
    n = 2_300_000  # > 2 loader chunks
    L = _two_iso_lines(n, seed=31)
    d = str(tmp_path) + "/"
    order = _write_files(d, L, [0, 8000, 20000])
    qa, gf = 0.7, 1.3
    with hkb.Context(0) as cf, _ctx_arrays(L, order, qa, gf) as ca:
        cf.set_options(qalphaL=qa, gammaF=gf)
        cf.load_species_file(d, "syn2", 0.0, 20000.0, 0, CUT)
        assert cf.num_lines == n
        assert np.array_equal(cf.line_order(), ca.line_order())
        for c in (cf, ca):
            c.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, CUT)
        for T, P in ((296.0, 1.0), (1700.0, 0.03)):
            a, b = cf.state_lines(T, P), ca.state_lines(T, P)
            for u, v in zip(a, b):
                assert np.array_equal(u, v)
            assert np.array_equal(cf.opacity([T], [P]), ca.opacity([T], [P]))


def test_species_file_selects_files_by_range(tmp_path):
    L = _two_iso_lines(60_000, seed=5)
    d = str(tmp_path) + "/"
    _write_files(d, L, [0, 5000, 10000, 15000, 20000])
    with hkb.Context(0) as c:
        # heliosk.cu:943-956: files whose range widened by the cut reaches [numin, numax]
        c.load_species_file(d, "syn2", 6000.0, 9000.0, 0, 25.0)
        assert c.num_lines == int(((L["nu"] >= 5000) & (L["nu"] < 10000)).sum())
        c.load_species_file(d, "syn2", 4990.0, 9000.0, 0, 25.0)
        assert c.num_lines == int((L["nu"] < 10000).sum())
        c.load_species_file(d, "syn2", 6000.0, 9000.0, 1, 25.0)  # cutMode 1 reads all files
        assert c.num_lines == 60_000


def test_species_file_unknown_isotopologue(tmp_path):
    L = _two_iso_lines(3000, seed=9)
    d = str(tmp_path) + "/"
    _write_files(d, L, [0, 8000, 20000])
    # overwrite one record id of the second file with an id outside the table
    f2 = os.path.join(d, "syn2_08000-20000.bin")
    rec = np.fromfile(f2, synth.HITRAN_DTYPE)
    rec["cid"][7] = b" 99"
    rec.tofile(f2)
    with hkb.Context(0) as c:
        with pytest.raises(hkb.HkError) as e:
            c.load_species_file(d, "syn2", 0.0, 20000.0, 0, CUT)
        assert e.value.status == -3
        assert "partition function not found. 7 | 99| 11|" in str(e.value)


def test_species_file_truncated(tmp_path):
    L = _two_iso_lines(5000, seed=3)
    d = str(tmp_path) + "/"
    _write_files(d, L, [0, 20000])
    f = os.path.join(d, "syn2.bin")
    raw = open(f, "rb").read()
    open(f, "wb").write(raw[: 68 * 4000 + 10])
    with hkb.Context(0) as c:
        with pytest.raises(hkb.HkError) as e:
            c.load_species_file(d, "syn2", 0.0, 20000.0, 0, CUT)
        assert e.value.status == -3 and "truncated (4000 of 5000 records)" in str(e.value)
        with pytest.raises(hkb.HkError) as e:
            c.load_species_file(d, "missing", 0.0, 20000.0, 0, CUT)
        assert e.value.status == -2


def test_exomol_file_equals_arrays(tmp_path):
    n = 1_500_000
    L = synth.exomol_lines(n, seed=12, nu_max=20000.0)
    L["A"] = np.random.default_rng(2).uniform(0.0, 50.0, n)
    d = str(tmp_path) + "/"
    synth.write_species(d, "exo", database=2, nfiles=1, nl=[n], limits=(0, 20000),
                        defaultL=0.07, defaultn=0.5)
    synth.write_exomol_bin(os.path.join(d, "exo.bin"), L)
    with hkb.Context(0) as cf, hkb.Context(0) as ca:
        cf.load_species_file(d, "exo", 0.0, 20000.0, 0, CUT)
        ca.set_species(hkb.EXOMOL, [synth.MASS], [1.0], defaultL=0.07, defaultn=0.5)
        T, Q = synth.q_table()
        ca.set_partition(0, T, Q)
        ca.load_lines_exomol(L)
        assert cf.num_lines == ca.num_lines == n
        for c in (cf, ca):
            c.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, CUT)
        a, b = cf.state_lines(1200.0, 0.1), ca.state_lines(1200.0, 0.1)
        for u, v in zip(a, b):
            assert np.array_equal(u, v)
        assert np.array_equal(cf.opacity([1200.0], [0.1]), ca.opacity([1200.0], [0.1]))
