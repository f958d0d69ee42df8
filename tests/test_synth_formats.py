"""Synthetic inputs are written in the reference's record layouts."""
import os

import numpy as np

from hkb import synth


def test_record_sizes_and_roundtrip(tmp_path):
    L = synth.hitran_lines(1000, seed=0)
    p = tmp_path / "x.bin"
    synth.write_hitran_bin(str(p), L)
    assert os.path.getsize(p) == 68 * 1000
    raw = p.read_bytes()
    assert raw[:4] == b" 11\x00"           # cid "%2d%s" (hitran.cpp:315)
    back = synth.read_hitran_bin(str(p))
    for k in ("nu", "S", "EL", "gair", "n"):
        assert np.array_equal(back[k], L[k])
    E = synth.exomol_lines(100, seed=4)
    q = tmp_path / "e.bin"
    synth.write_exomol_bin(str(q), E)
    assert os.path.getsize(q) == 32 * 100


def test_workload_distributions():
    L = synth.hitran_lines(200000, seed=0)
    assert 0 <= L["nu"].min() and L["nu"].max() <= 30000
    assert abs(L["EL"].mean() - 3000) < 50
    assert 0.01 <= L["gair"].min() and L["gair"].max() <= 0.1
    assert 0.4 <= L["n"].min() and L["n"].max() <= 0.8
    s296 = L["S"] * (synth.MASS / synth.NA) / synth.q_of_T(296.0)
    lg = np.log10(s296)
    assert -30.0 <= lg.min() and lg.max() <= -18.0
    T, P = synth.table_states()
    assert len(T) == 600 and T.min() == 100.0 and abs(T.max() - 3000.0) < 1e-9
    assert abs(np.log10(P.min()) + 8) < 1e-12 and abs(np.log10(P.max()) - 3) < 1e-12


def test_species_file_layout(tmp_path):
    synth.write_species(str(tmp_path), "syn", database=0, nl=[10])
    txt = (tmp_path / "syn.param").read_text().splitlines()
    assert txt[0] == "Database = 0"
    assert txt[3] == "Number of Isotopologues = 1"
    q = np.loadtxt(tmp_path / "q_synth.txt")
    assert q.shape == (5000, 2)
    assert q[999, 1] == 0.1 * 1000.0 ** 1.5
