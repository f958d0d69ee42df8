"""Run a HELIOS-K executable on a synthetic run directory.

MEASUREMENT / TEST INFRASTRUCTURE.  Two executables read the same inputs
(param.dat, <species>.param, partition file, binary line file):
  * oracle/_ref/heliosk -- the reference's own CUDA build (oracle/Makefile
    target `ref`; built here, never part of the product), timed beside this
    library in bench.py;
  * helios-k_b200/bin/heliosk -- this library's drop-in executable, whose
    outputs the tests compare with the reference's formats and the oracle.
The run writes Out_<name>.bin (float K, doStoreFullK = 2) and
Out_<name>_cbin.dat (Chebyshev coefficients per bin, doResampling = 1).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(_HERE)
REF_EXE = os.path.join(_HERE, "_ref", "heliosk")
OUR_EXE = os.path.join(ROOT, "helios-k_b200", "bin", "heliosk")
sys.path.insert(0, os.path.join(ROOT, "helios-k_b200"))


def write_data(data_dir, lines, species="syn"):
    """A HITRAN-format species in data_dir: <species>.param (one
    isotopologue), its partition file and one binary line file."""
    from hkb import synth
    os.makedirs(data_dir, exist_ok=True)
    synth.write_species(data_dir, species, database=0, nfiles=1, nl=[len(lines["nu"])],
                        limits=(int(np.floor(np.min(lines["nu"]))), int(np.ceil(np.max(lines["nu"]))) + 1))
    synth.write_hitran_bin(os.path.join(data_dir, species + ".bin"), lines)


def write_run(d, data_dir, T, P, numin, numax, dnu, cut, nbins, nC, name="syn", species="syn",
              store_k=2, resample=1, tuning=1, **extra):
    """param.dat for one T and one P (or, P a list, a PFile of pressures) in
    run directory d, reading data_dir; extra: more param.dat keys (spaces
    as underscores), e.g. doMean=1, doTransmission=1, nTr=100, dTr=0.05."""
    from hkb import synth
    os.makedirs(d, exist_ok=True)
    pfile = "-"
    if np.ndim(P) > 0:
        pfile = os.path.join(d, "P.dat")
        with open(pfile, "w") as f:
            f.write("\n".join("%.17g" % v for v in P) + "\n")
        P = float(P[0])
    synth.write_param(os.path.join(d, "param.dat"), name=name, T=T, P=P, PFile=pfile,
                      Species_Name=species, pathToData=data_dir.rstrip("/") + "/", numin=numin,
                      numax=numax, dnu=dnu, cut=cut, nbins=nbins, nC=nC,
                      doResampling=resample, doStoreFullK=store_k, doTuning=tuning, **extra)


def make_run_dir(d, lines, T, P, numin, numax, dnu, cut, nbins, nC, name="syn",
                 species="syn", store_k=2, resample=1, tuning=1, **extra):
    """Species data and param.dat together in directory d."""
    write_data(d, lines, species)
    write_run(d, d, T, P, numin, numax, dnu, cut, nbins, nC, name, species, store_k, resample,
              tuning, **extra)


_TIME_RE = {
    "input_s": re.compile(r"Time for input total:\s+([0-9.eE+-]+)"),
    "lines_s": re.compile(r"Time for Lines total:\s+([0-9.eE+-]+)"),
    "kx_s": re.compile(r"Time for K\(x\) total:\s+([0-9.eE+-]+)"),
}


def run(exe, d, timeout=600):
    """Run exe in d; returns dict(rc, wall_s, the reference's reported
    totals (input_s, lines_s, kx_s) when printed, tail of the output)."""
    t0 = time.perf_counter()
    p = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=timeout)
    out = {"rc": p.returncode, "wall_s": time.perf_counter() - t0,
           "tail": (p.stdout + p.stderr)[-2000:]}
    for k, r in _TIME_RE.items():
        m = r.findall(p.stdout)
        out[k] = float(m[-1]) if m else None
    out["info"] = info_times(d)
    return out


def info_times(d, name="syn"):
    """'Time for ...: x seconds' entries of Info_<name>.dat (both executables
    write the reference's Info layout); the last value of each kind."""
    out = {}
    try:
        with open(os.path.join(d, "Info_%s.dat" % name)) as f:
            for ln in f:
                m = re.match(r"\s*Time for ([^:]+):\s+([0-9.eE+-]+)", ln)
                if m:
                    out[m.group(1).strip()] = float(m.group(2))
    except OSError:
        pass
    return out


def read_k(d, name="syn"):
    return np.fromfile(os.path.join(d, "Out_%s.bin" % name), np.float32)


def read_cbin(d, name="syn"):
    """Out_<name>_cbin.dat rows: kmin, ystart, nC coefficients."""
    rows = []
    with open(os.path.join(d, "Out_%s_cbin.dat" % name)) as f:
        for ln in f:
            v = ln.split()
            if v:
                rows.append([float(t) for t in v])
    return np.array(rows)
