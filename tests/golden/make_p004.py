"""Regenerate tests/golden/p004.npz from the reference's shipped run plots/p004.

The reference ships one self-consistent k-distribution run (HELIOS-K
plots/p004, 30000 grid points, one bin, nC = 20):
  Out_i.dat      full K(x) of run "i"            -> K_i
  Out_i_bin.dat  per-bin sorted K of run "i"     -> Ksorted_i
  Out_r.dat      full K(x) of run "r"            -> K_r
  Out_r_cbin.dat Chebyshev fit of run "r"        -> cbin_r (kmin, ystart, c0..c19)
  Out_r_bin.dat  reconstruction from the fit     -> Krecon_r
The text values are printed with %.20g, so parsing them as float64 is exact.

p004_files.json records the files the reference's own run wrote, to pin the
drop-in's output files to them: the SHA-256, size and line count of
Out_i_bin.dat and Out_r_bin.dat, the SHA-256 of Out_r_bin.dat's first column
(the "%g" bin coordinates), and the whole text of Out_r_cbin.dat.

Usage (needs the reference source tree; the fixtures themselves are committed):
  python tests/golden/make_p004.py /path/to/HELIOS-K
  (or HK_REFERENCE_DIR=/path/to/HELIOS-K python tests/golden/make_p004.py)
"""
import hashlib
import json
import os
import sys

import numpy as np


def _two_col(path):
    rows = [ln.split() for ln in open(path) if ln.strip()]
    a = np.array([[float(v) for v in r[:2]] for r in rows], dtype=np.float64)
    return a[:, 0], a[:, 1]


def main(ref_root):
    d = os.path.join(ref_root, "plots", "p004")
    x_i, K_i = _two_col(os.path.join(d, "Out_i.dat"))
    y_i, Ks_i = _two_col(os.path.join(d, "Out_i_bin.dat"))
    x_r, K_r = _two_col(os.path.join(d, "Out_r.dat"))
    y_r, Kr_r = _two_col(os.path.join(d, "Out_r_bin.dat"))
    cb = np.array([float(v) for v in open(os.path.join(d, "Out_r_cbin.dat")).read().split()],
                  dtype=np.float64)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "p004.npz")
    np.savez_compressed(out, x_i=x_i, K_i=K_i, Ksorted_i=Ks_i, x_r=x_r, K_r=K_r,
                        Krecon_r=Kr_r, cbin_r=cb,
                        params=np.array([0.0, 30000.0, 1.0, 1, 20, 0.0]))
    print("wrote", out, len(K_i), len(cb))
    files = {}
    for name in ("Out_i_bin.dat", "Out_r_bin.dat"):
        raw = open(os.path.join(d, name), "rb").read()
        col0 = b"\n".join(ln.split(b" ")[0] for ln in raw.split(b"\n") if ln.strip())
        files[name] = {"sha256": hashlib.sha256(raw).hexdigest(), "bytes": len(raw),
                       "lines": raw.count(b"\n"), "col0_sha256": hashlib.sha256(col0).hexdigest()}
    files["Out_r_cbin.dat"] = {"text": open(os.path.join(d, "Out_r_cbin.dat")).read()}
    jout = os.path.join(os.path.dirname(os.path.abspath(__file__)), "p004_files.json")
    with open(jout, "w") as f:
        json.dump(files, f, indent=1)
    print("wrote", jout)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HK_REFERENCE_DIR")
    if not root:
        sys.exit("usage: make_p004.py <reference source tree> (or set HK_REFERENCE_DIR)")
    main(root)
