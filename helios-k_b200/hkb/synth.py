"""Seeded synthetic line lists with the shapes of the benchmark workloads.

No real line list ships with the reference, so every workload uses seeded
synthetic data with the stated distributions, written (optionally) in the
reference's own file formats so the same inputs feed every implementation:
  * <name>.param species file (ISO.h:16-219 layout),
  * a 2-column partition file Q(T) = 0.1 T^1.5 on a 1 K grid, 1..5000 K,
  * HITRAN 68-byte records (hitran.cpp:406-414) or ExoMol 32-byte records
    (prepareExomol.cpp:222-225).
The file strength follows hitran.cpp:401-402: S_file = S(296) Q(296) / (m / NA).

Workloads (seed = index unless stated):
  small    1e5 lines, nu0 ~ U[0,30000], log10 S ~ U[-30,-18], E'' ~ Exp(3000),
           gamma_air ~ U[0.01,0.1], n ~ U[0.4,0.8]; T=1000 K, P=1 atm;
           grid 0-30000 dnu 0.01; cut 100; 300 bins; nC 20.
  hitemp   1e7 lines, same but log10 S ~ U[-32,-18]; T=1500 K, P=0.1 atm; cut 25.
  table    the hitemp list on 20 T (100-3000 K, linear) x 30 P (1e-8-1e3 atm, log).
  adjoint  1e6 lines (small distributions), grid 1000-10000, T=800 K, P=1 atm.
  exomol   5e8 lines, nu0 ~ U[0,40000], log10 S ~ U[-40,-18], E'' ~ Exp(8000),
           gamma_L = 0.07, n = 0.5; 4x4 T (500-2500) x P (1e-4-10, log);
           grid 0-40000 dnu 0.01, cut 25, 400 bins.
"""
from __future__ import annotations

import os

import numpy as np

NA = 6.0221412927e23
MASS = 18.0


def q_of_T(T):
    return 0.1 * np.asarray(T, dtype=np.float64) ** 1.5


def q_table():
    T = np.arange(1, 5001, dtype=np.float64)
    return T, q_of_T(T)


def hitran_lines(n, seed=0, logS=(-30.0, -18.0), nu_max=30000.0, E_mean=3000.0,
                 nu_min=0.0):
    """Line dict (nu, S_file, EL, A, delta, gair, gself, n, iso) in file units."""
    rng = np.random.default_rng(seed)
    nu = rng.uniform(nu_min, nu_max, n)
    S296 = 10.0 ** rng.uniform(logS[0], logS[1], n)
    EL = rng.exponential(E_mean, n)
    gair = rng.uniform(0.01, 0.1, n)
    nexp = rng.uniform(0.4, 0.8, n)
    S_file = S296 * float(q_of_T(296.0)) / (MASS / NA)
    z = np.zeros(n)
    return dict(nu=nu, S=S_file, EL=EL, A=z.copy(), delta=z.copy(), gair=gair,
                gself=gair.copy(), n=nexp, iso=np.zeros(n, np.int32))


def exomol_lines(n, seed=4, logS=(-40.0, -18.0), nu_max=40000.0, E_mean=8000.0,
                 chunk=1 << 24):
    """ExoMol-format dict (nu, S_file, EL, A) drawn in chunks of `chunk` lines
    (bounded host temporaries for 5e8-line lists); widths come from the
    species defaults."""
    rng = np.random.default_rng(seed)
    nu = np.empty(n)
    S_file = np.empty(n)
    EL = np.empty(n)
    f = float(q_of_T(296.0)) / (MASS / NA)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        nu[a:b] = rng.uniform(0.0, nu_max, b - a)
        S_file[a:b] = 10.0 ** rng.uniform(logS[0], logS[1], b - a) * f
        EL[a:b] = rng.exponential(E_mean, b - a)
    return dict(nu=nu, S=S_file, EL=EL, A=np.zeros(n))


WORKLOADS = {
    "small": dict(n=100_000, seed=0, logS=(-30.0, -18.0), T=[1000.0], P=[1.0],
                  numin=0.0, numax=30000.0, dnu=0.01, cut=100.0, nbins=300, nC=20),
    "hitemp": dict(n=10_000_000, seed=1, logS=(-32.0, -18.0), T=[1500.0], P=[0.1],
                   numin=0.0, numax=30000.0, dnu=0.01, cut=25.0, nbins=300, nC=20),
    "adjoint": dict(n=1_000_000, seed=3, logS=(-30.0, -18.0), T=[800.0], P=[1.0],
                    numin=1000.0, numax=10000.0, dnu=0.01, cut=100.0, nbins=300, nC=20),
    # the hitemp line distribution at 1/10 of the line density over the same
    # grid (used for profiler captures: same tiles and per-pair mix, 1/10 of
    # the work, ~150 MB on the device)
    # 5e8 ExoMol-format lines (~12 GB of line columns in HBM), 4 x 4 states
    "exomol": dict(n=500_000_000, seed=4, logS=(-40.0, -18.0), numin=0.0, numax=40000.0,
                   dnu=0.01, cut=25.0, nbins=400, nC=20, database="exomol", defaultL=0.07,
                   defaultn=0.5, nu_max=40000.0, E_mean=8000.0),
    "hitemp_sparse": dict(n=1_000_000, seed=1, logS=(-32.0, -18.0), T=[1500.0], P=[0.1],
                          numin=0.0, numax=30000.0, dnu=0.01, cut=25.0, nbins=300, nC=20),
}


def table_states():
    """20 temperatures x 30 pressures (the T-P table workload)."""
    Ts = 100.0 + np.arange(20) * (2900.0 / 19.0)
    Ps = 10.0 ** (-8.0 + np.arange(30) * (11.0 / 29.0))
    TT, PP = np.meshgrid(Ts, Ps, indexing="ij")
    return TT.ravel(), PP.ravel()


def exomol_states():
    Ts = np.linspace(500.0, 2500.0, 4)
    Ps = 10.0 ** np.linspace(-4.0, 1.0, 4)
    TT, PP = np.meshgrid(Ts, Ps, indexing="ij")
    return TT.ravel(), PP.ravel()


# ------------------------------------------------------------- file writers

def write_species(dirname, name, database=0, nfiles=1, nl=None, limits=(0, 30000),
                  defaultL=0.0, defaultn=0.0, qfile="q_synth.txt", npfcol=2, isos=None):
    """<name>.param in the layout ISO.h:16-219 parses.  isos: rows
    (cid, abundance, molar mass), all on the synthetic partition table;
    default one isotopologue of mass MASS."""
    os.makedirs(dirname, exist_ok=True)
    nl = list(nl or [0])
    if isos is None:
        isos = [("11" if database in (0, 1) else "0", 1.0, MASS)]
    lines = [
        f"Database = {database}",
        "Molecule number = 1",
        f"Name = {name}",
        f"Number of Isotopologues = {len(isos)}",
        "#ID Abundance      Q(296K)   g     Molar Mass(g)  partition file :",
        *[f"{cid} {ab:.10g} {float(q_of_T(296.0)):.10g} 1 {m:.6f} {qfile}" for cid, ab, m in isos],
        f"Number of columns in partition File = {npfcol}",
        f"Number of line/transition files = {nfiles}",
        "Number of lines per file :",
        *[str(int(v)) for v in nl],
        "Line file limits :",
        *[str(int(v)) for v in limits],
        "#ExoMol :",
        "Number of states = 0",
        "Number of columns in transition files = 0",
        f"Default value of Lorentzian half-width for all lines = {defaultL:g}",
        f"Default value of temperature exponent for all lines = {defaultn:g}",
        "Version = 0",
    ]
    with open(os.path.join(dirname, name + ".param"), "w") as f:
        f.write("\n".join(lines) + "\n")
    T, Q = q_table()
    with open(os.path.join(dirname, qfile), "w") as f:
        for t, q in zip(T, Q):
            f.write(f"{int(t)} {q:.17g}\n")


HITRAN_DTYPE = np.dtype([("cid", "S4"), ("nu", "<f8"), ("S", "<f8"), ("EL", "<f8"),
                         ("A", "<f8"), ("delta", "<f8"), ("gair", "<f8"),
                         ("gself", "<f8"), ("n", "<f8")])
EXOMOL_DTYPE = np.dtype([("nu", "<f8"), ("S", "<f8"), ("EL", "<f8"), ("A", "<f8")])
assert HITRAN_DTYPE.itemsize == 68 and EXOMOL_DTYPE.itemsize == 32


def write_hitran_bin(path, lines, cids=None):
    """68-byte records; cids: per-record 3-character isotopologue ids
    (default " 11" for every line)."""
    rec = np.empty(len(lines["nu"]), HITRAN_DTYPE)
    rec["cid"] = b" 11" if cids is None else cids
    for k in ("nu", "S", "EL", "A", "delta", "gair", "gself", "n"):
        rec[k] = lines[k]
    rec.tofile(path)


def write_exomol_bin(path, lines):
    rec = np.empty(len(lines["nu"]), EXOMOL_DTYPE)
    for k in ("nu", "S", "EL", "A"):
        rec[k] = lines[k]
    rec.tofile(path)


def read_hitran_bin(path):
    rec = np.fromfile(path, HITRAN_DTYPE)
    return {k: rec[k].astype(np.float64) for k in ("nu", "S", "EL", "A", "delta", "gair",
                                                   "gself", "n")}


def write_param(path, **kv):
    """param.dat in the key order of the reference's example (host.h:95-299)."""
    keys = [("name", "syn"), ("T", 1000.0), ("P", 1.0), ("PFile", "-"),
            ("Species Name", "syn"), ("SpeciesFile", "-"), ("ciaSystem", "-"),
            ("pathToData", ""), ("numin", 0.0), ("numax", 30000.0), ("dnu", 0.01),
            ("Nnu per bin", 0), ("cutMode", 0), ("cut", 100.0), ("doResampling", 0),
            ("nC", 20), ("doTransmission", 0), ("nTr", 1000), ("dTr", 0.05),
            ("doStoreFullK", 1), ("pathToK", ""), ("doStoreSK", 0), ("nbins", 300),
            ("binsFile", "-"), ("OutputEdgesFile", "-"), ("kmin", 0.0), ("qalphaL", 1.0),
            ("gammaF", 1.0), ("doMean", 0), ("Units", 0), ("ReplaceFiles", 1),
            ("profile", 1), ("doTuning", 1)]
    # optional keys (host.h:95-299), written only when given
    optional = ["removePlinth", "subLorentzianfile"]
    with open(path, "w") as f:
        for k, default in keys:
            v = kv.get(k.replace(" ", "_"), kv.get(k, default))
            f.write(f"{k} = {v}\n")
        for k in optional:
            if k in kv:
                f.write(f"{k} = {kv[k]}\n")


# ------------------------------------------------------------ CIA files

def write_cia(path, sets, formula="H2-H2"):
    """A HITRAN-format CIA file (Richard et al. 2012): per temperature set a
    100-character header -- formula (20), numin (10), numax (10), number of
    points (7), T (7), max cross section (10), resolution (6), comment (27),
    reference (3) -- then "nu cia" rows.  sets: [(T, nu array, cia array)]."""
    with open(path, "w") as f:
        for T, nu, cia in sets:
            nu = np.asarray(nu, np.float64)
            cia = np.asarray(cia, np.float64)
            # readers stop a set where the last nu equals the header's numax
            # (host.h:749): both must print to the same value
            if float(f"{nu[-1]:10.3f}") != float(f"{nu[-1]:10.4f}"):
                raise ValueError("the last nu of a set must have at most 3 decimals")
            f.write(f"{formula:>20s}{nu[0]:10.3f}{nu[-1]:10.3f}{len(nu):7d}{T:7.1f}"
                    f"{cia.max():10.3e}{0.0:6.3f}{'synthetic':>27s}{1:3d}\n")
            for a, b in zip(nu, cia):
                f.write(f"{a:10.4f} {b:10.3e}\n")
