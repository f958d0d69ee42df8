"""GPU: the drop-in executable pinned to the files the reference's own run
wrote (HELIOS-K plots/p004: T = 500 K, one bin of 30000 points, dnu = 1,
nC = 20; fixtures tests/golden/p004.npz and p004_files.json, both made by
tests/golden/make_p004.py from the reference's files).

With doStoreFullK = -1 the executable reads K back from Out_<name>.dat
instead of computing it (heliosk.cu:1860-1935), so the per-bin sort, the fit
and the writers (heliosk.cu:2046-2193, 2222-2355) run on the reference's own
K through the real process contract (param.dat in, Out_* files out):
  run i (doResampling 0, doStoreSK 1): Out_i_bin.dat byte-identical to the
    reference's file (the sorted values are bit-exact, the formats "%g" and
    "%.20g" are the reference's);
  run r (doResampling 1, doStoreSK 1): Out_r_cbin.dat with the reference's
    kmin and ystart text and layout, coefficients within 1e-9 absolute;
    Out_r_bin.dat with the reference's line count and byte-identical bin
    coordinates, reconstructed K within 1e-9 relative.
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_run  # noqa: E402
from hkb import synth  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def files():
    with open(os.path.join(ROOT, "tests", "golden", "p004_files.json")) as f:
        return json.load(f)


def _run(d, g, name, resample):
    """param.dat of p004's run `name` reading K from Out_<name>.dat in d."""
    K = g["K_" + name]
    x = g["x_" + name]
    with open(os.path.join(d, f"Out_{name}.dat"), "w") as f:
        f.writelines("%.20g %.20g\n" % (a, b) for a, b in zip(x, K))
    synth.write_param(os.path.join(d, "param.dat"), name=name, T=500.0, P=1.0,
                      Species_Name="syn", pathToData=d.rstrip("/") + "/", numin=0.0,
                      numax=30000.0, dnu=1.0, cutMode=0, cut=25.0, doResampling=resample,
                      nC=20, doStoreFullK=-1, pathToK=d.rstrip("/") + "/", doStoreSK=1, nbins=1,
                      kmin=0.0, qalphaL=1.0, doTuning=1)
    r = ref_run.run(ref_run.OUR_EXE, d, timeout=300)
    assert r["rc"] == 0, r["tail"]


def test_dropin_sorted_bins_byte_identical(tmp_path, golden_p004, files):
    assert os.path.exists(ref_run.OUR_EXE), "build helios-k_b200/bin/heliosk first"
    d = str(tmp_path)
    # a species file only for the mean molar mass (Units = 0: no effect)
    synth.write_species(d, "syn", database=0, nfiles=1, nl=[0])
    _run(d, golden_p004, "i", 0)
    raw = open(os.path.join(d, "Out_i_bin.dat"), "rb").read()
    want = files["Out_i_bin.dat"]
    assert len(raw) == want["bytes"] and raw.count(b"\n") == want["lines"]
    assert hashlib.sha256(raw).hexdigest() == want["sha256"]


def test_dropin_fit_files_match_reference(tmp_path, golden_p004, files):
    assert os.path.exists(ref_run.OUR_EXE), "build helios-k_b200/bin/heliosk first"
    d = str(tmp_path)
    synth.write_species(d, "syn", database=0, nfiles=1, nl=[0])
    _run(d, golden_p004, "r", 1)
    ours = open(os.path.join(d, "Out_r_cbin.dat")).read()
    ref = files["Out_r_cbin.dat"]["text"]
    assert ours.endswith(" \n\n") and ref.endswith(" \n\n")
    to, tr = ours.split(), ref.split()
    assert len(to) == len(tr) == 22
    assert to[:2] == tr[:2]  # kmin "0", ystart = Nxmin / (Nxb - 1) to the last digit
    err = np.max(np.abs(np.array(to[2:], float) - np.array(tr[2:], float)))
    print(f"p004 cbin: coefficients max abs difference {err:.2e}")
    assert err < 1e-9
    raw = open(os.path.join(d, "Out_r_bin.dat"), "rb").read()
    want = files["Out_r_bin.dat"]
    assert raw.count(b"\n") == want["lines"] and raw.endswith(b"\n\n\n")
    rows = [ln.split(b" ") for ln in raw.split(b"\n") if ln.strip()]
    col0 = b"\n".join(r[0] for r in rows)
    assert hashlib.sha256(col0).hexdigest() == want["col0_sha256"]
    K = np.array([float(r[1]) for r in rows])
    R = golden_p004["Krecon_r"]
    nz = R != 0
    assert np.array_equal(K[~nz], R[~nz])
    rel = np.max(np.abs(K[nz] - R[nz]) / R[nz])
    print(f"p004 reconstruction max rel difference {rel:.2e}")
    assert rel < 1e-9
