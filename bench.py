#!/usr/bin/env python
"""Benchmark of the HELIOS-K opacity hot path on B200.

One step = one pass of the path over one batch: the line scaling and Voigt
line sum of every state onto the grid followed by the per-bin sort +
Chebyshev k-distribution fit, replayed as one CUDA graph (hk_table_run).
Inputs are resident in HBM (line list >> L2, so no L2 flush is needed
between steps).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload hitemp|small|table|...] [--precision mixed|plain]

Metric: Voigt evaluations per second (algorithmic (line, grid point) pairs
inside the cutoff windows, counted exactly from the index windows), plus the
seconds per state and per T-P table.  The default run (hitemp: one state of
a 1e7-line list) adds a table leg: the 600-state T-P table of the same list
as one graph replay (s_per_table), its plain-FP64 subset, its error against
the FP64 oracle and the reference's own CUDA build on one temperature row.

Multi-GPU (one process per GPU): every rank computes its own copy of the
single-state workload (weak scaling; time = max over ranks, value = pairs of
all ranks / that time); the table leg splits the table's states across the
ranks (rank r takes states r, r + N, ...; no collective on the data path).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "helios-k_b200"))

# algorithmic FP32 flops per pair by region (committed constants; the C-region
# figure grows with the Algorithm 916 series length n_iter).  Each constant
# already holds the accumulate FMA (region A: offset, r^2, rcp, accumulate);
# the sums carry no Kahan compensation, so no per-pair term is added.
F_A, F_B, F_C0, F_C_ITER = 6, 20, 30, 12
# DRAM bytes (read + write) of one voigt_sum_kernel<1> launch, from one ncu
# capture of this workload (profiles/dram_traffic_hitemp.txt); other
# workloads have no capture and report null
VOIGT_DRAM_BYTES = {"hitemp-1e7-lines-single-state": 2007904000 + 110621952}
SIZEOF_STATE = 2672  # bytes of hkb::StateDev copied per state per call


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hitemp",
                    choices=["hitemp", "small", "table", "table_sparse", "hitemp_sparse", "adjoint",
                             "exomol"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "plain"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-FP64 comparison leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip timing the reference's own CUDA build beside ours")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-table", action="store_true",
                    help="skip the T-P table leg of the default (hitemp) run")
    ap.add_argument("--no-fused", action="store_true",
                    help="skip timing the table as one persistent launch (table mode 1)")
    ap.add_argument("--table-steps", type=int, default=1,
                    help="timed replays of the 600-state table (each ~17 s), after 1 untimed")
    ap.add_argument("--table-mode", type=int, default=0, choices=[0, 1],
                    help="table graph of the main workload: 0 per-batch launches, 1 one persistent launch")
    ap.add_argument("--tuning", type=int, default=2, choices=[0, 1, 2],
                    help="tile-shape tuner: 0 fixed default shape, 1 when it pays, 2 once "
                         "before the timed steps")
    return ap.parse_args()


def workload(name):
    from hkb import synth
    if name == "table":
        W = dict(synth.WORKLOADS["hitemp"])
        T, P = synth.table_states()
        W["T"], W["P"] = list(T), list(P)
        W["label"] = "tp-table-1e7-lines-600-states"
    elif name == "table_sparse":
        # 20 states spread over the T-P table on a 1e6-line list: K (20 x 3e6
        # FP64, 480 MB) is larger than L2, the line records 2.2 GB -- the
        # profiling case of the line prep and the per-bin sort/fit
        W = dict(synth.WORKLOADS["hitemp_sparse"])
        T, P = synth.table_states()
        sub = np.linspace(0, len(T) - 1, 20).astype(int)
        W["T"], W["P"] = list(np.asarray(T)[sub]), list(np.asarray(P)[sub])
        W["label"] = "tp-subtable-1e6-lines-20-states"
    elif name == "exomol":
        W = dict(synth.WORKLOADS["exomol"])
        T, P = synth.exomol_states()
        W["T"], W["P"] = list(T), list(P)
        W["label"] = "exomol-5e8-lines-4x4-states"
    else:
        W = dict(synth.WORKLOADS[name])
        W["label"] = {"hitemp": "hitemp-1e7-lines-single-state",
                      "small": "small-1e5-lines-single-state",
                      "adjoint": "adjoint-1e6-lines-1000-10000cm-1",
                      "hitemp_sparse": "hitemp-distribution-1e6-lines-single-state"}[name]
    return W


def make_lines(W):
    from hkb import synth
    if W.get("database") == "exomol":
        return synth.exomol_lines(W["n"], seed=W["seed"], logS=W["logS"], nu_max=W["nu_max"],
                                  E_mean=W["E_mean"])
    return synth.hitran_lines(W["n"], seed=W["seed"], logS=W["logS"],
                              nu_min=W.get("nu_min", 0.0), nu_max=W.get("nu_max", 30000.0))


def open_ctx(W, L, device):
    import hkb
    from hkb import synth
    ctx = hkb.Context(device)
    Tq, Qq = synth.q_table()
    if W.get("database") == "exomol":
        ctx.set_species(hkb.EXOMOL, [synth.MASS], [1.0], W["defaultL"], W["defaultn"])
        ctx.set_partition(0, Tq, Qq)
        ctx.load_lines_exomol(L)
    else:
        ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
        ctx.set_partition(0, Tq, Qq)
        ctx.set_options(qalphaL=1.0)
        ctx.load_lines_hitran(L)
    ctx.set_grid(W["numin"], W["numax"], W["dnu"], W["nbins"], 0, W["cut"])
    return ctx


def count_pairs(ctx, T, P):
    """Exact (A, B, C) pair counts of one state from the device index windows."""
    return ctx.count_pairs(T, P)


def c_series_iterations(ctx, T, P, sample=1000, seed=0):
    """Mean Algorithm-916 series length of the reference's FP32 form over
    region-C pairs (the n_iter of the flop model), replaying its stopping rule
    (|delta s| < TOLF for s1, s2, s3) in numpy on a sample of lines."""
    rng = np.random.default_rng(seed)
    nu, S, iad, vy, win = ctx.state_lines(T, P)
    has = np.nonzero(win[:, 3] > win[:, 2])[0]
    if len(has) == 0:
        return 0.0
    ls = rng.choice(has, size=min(sample, len(has)))
    a = np.float32(0.5999962687492371)
    tol = np.float32(2.48e-12)
    its = []
    for l in ls:
        i = rng.integers(win[l, 2], win[l, 3])
        x = np.float32(abs((ctx._numin + i * ctx._dnu - nu[l]) * iad[l]))
        y = np.float32(vy[l])
        if x == 0 or y == 0:
            its.append(0)
            continue
        n0 = int(np.ceil(x / a))
        s = np.zeros(3, np.float32)
        old = np.zeros(3, np.float32)
        stop = [False] * 3
        n_it = 0
        for n in range(1, 100):
            n_it = n
            an, ap, am = a * n, a * (n0 + n - 1), a * (n0 - n)
            yy = y * y
            s[0] += np.float32(1) / (an * an + yy) * np.exp(-(an * an + x * x))
            s[1] += np.float32(1) / (an * an + yy) * np.exp(-(an + x) * (an + x))
            s[2] += np.float32(1) / (ap * ap + yy) * np.exp(-(ap - x) * (ap - x))
            if n0 - n >= 1:
                s[2] += np.float32(1) / (am * am + yy) * np.exp(-(am - x) * (am - x))
            for k in range(3):
                if abs(s[k] - old[k]) < tol:
                    stop[k] = True
            if all(stop):
                break
            old[:] = s
        its.append(n_it)
    return float(np.mean(its))


class Clocks:
    """SM clock and clock-event reasons sampled during the timed region:
    NVML read every 10 ms from a thread (read-only queries), else
    nvidia-smi at 200 ms.  The NVML device is the CUDA device's (matched by
    UUID, else by index)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.p = None
        self.f = None
        self.thread = None
        self.nv = None
        self.handle = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.handle = self._nvml_handle(device)
        except Exception:
            self.nv = None

    def _nvml_handle(self, device):
        nv = self.nv
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(device).uuid)
            return nv.nvmlDeviceGetHandleByUUID("GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(device)

    def _poll(self):
        nv, h = self.nv, self.handle
        bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append(float(sm))
                for k, b in enumerate(bits):
                    if r & b:
                        self.reasons.add(self.NAMES[k])
            except Exception:
                pass
            self.stop_flag.wait(0.01)

    def start(self):
        if self.nv is not None:
            import threading
            self.samples, self.reasons = [], set()
            self.stop_flag = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join()
            self.thread = None
            smax = None
            try:
                smax = float(self.nv.nvmlDeviceGetMaxClockInfo(self.handle, self.nv.NVML_CLOCK_SM))
            except Exception:
                pass
            sm = self.samples
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                    "reasons": sorted(self.reasons), "samples": len(sm), "source": "nvml 10 ms"}
        if self.p is None:
            if self.f is not None:
                os.unlink(self.f.name)
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for k, nm in enumerate(self.NAMES):
                    if r[5 + k].strip() == "Active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi 200 ms"}


def dist_setup(args=None):
    """One process per GPU (torchrun env); NCCL on GPUs, gloo without them
    (HKB_DIST_BACKEND overrides).  States are independent, so the only
    collective is the max of the per-rank times."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    lrank = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = os.environ.get("HKB_DIST_BACKEND",
                                 "nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(lrank)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, lrank


def barrier_max(ws, value):
    """max over ranks of a per-rank time (the bench's only collective)."""
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_states(n, ws, rank):
    """The states of a table that rank `rank` of `ws` computes: r, r + ws,
    ... (disjoint; every state exactly once over the ranks; counts differ by
    at most one)."""
    return np.arange(rank, n, ws)


def workload_config(W):
    """The workload part of the JSON line: the same dict in both arms."""
    ns = len(W["T"])
    return {"workload": W["label"], "lines": W["n"],
            "grid_points": int(round((W["numax"] - W["numin"]) / W["dnu"])),
            "states": ns,
            "T": W["T"][0] if ns == 1 else f"{min(W['T']):g}-{max(W['T']):g} K x {len(set(W['T']))}",
            "P": W["P"][0] if ns == 1 else f"{min(W['P']):.3g}-{max(W['P']):.3g} atm x {len(set(W['P']))}",
            "cut_cm-1": W["cut"], "nbins": W["nbins"], "nC": W["nC"],
            "format": W.get("database", "hitran"),
            "l2": f"inputs larger than L2 (line columns ~{W['n'] * 48 / 1e9:.2g} GB resident), no flush"}


TILE = 2048  # points per sampled grid tile (oracle samples and parity)


def tile_order(nx, seed):
    """Seeded order in which the oracle samples grid tiles."""
    return [int(t) for t in np.random.default_rng(seed).permutation((nx + TILE - 1) // TILE)]


def oracle_state(W, L, T, P):
    """FP64 oracle line state and windows of one state (prep + index rule)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from hkb import synth
    Tq, Qq = synth.q_table()
    Q = oracle.partition(Tq, Qq, T)
    if W.get("database") == "exomol":
        nu, S, iad, vy = oracle.prep_exomol(L, synth.MASS, 1.0, Q, W["defaultL"], W["defaultn"], T, P)
    else:
        nu, S, iad, vy = oracle.prep_hitran(L, [synth.MASS], [1.0], [Q], T, P, qalphaL=1.0)
    nx = oracle.grid_nx(W["numin"], W["numax"], W["dnu"])
    win = oracle.windows(nu, S, iad, vy, W["numin"], W["dnu"], nx, 0, W["cut"])
    return nu, S, iad, vy, win, nx


def barrier_sum(ws, value):
    """sum over ranks of a per-rank count (outside the timed regions)."""
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def oracle_tiles_near(W, L, T, P, tiles):
    """The FP64 oracle's K on grid tiles of a list too large to prepare on the
    host: each tile from the lines whose cutoff windows can reach it (centres
    within cut + 1 cm^-1 of the tile; cutMode 0 and no pressure shift for the
    ExoMol format)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    nx = oracle.grid_nx(W["numin"], W["numax"], W["dnu"])
    out = {}
    for t in tiles:
        ib, ie = int(t * TILE), int(min(nx, (t + 1) * TILE))
        lo = W["numin"] + ib * W["dnu"] - W["cut"] - 1.0
        hi = W["numin"] + (ie - 1) * W["dnu"] + W["cut"] + 1.0
        sel = (L["nu"] > lo) & (L["nu"] < hi)
        Ls = {k: v[sel] for k, v in L.items()}
        nu, S, iad, vy, win, _ = oracle_state(W, Ls, T, P)
        out[t], _ = oracle.opacity(nu, S, iad, vy, win, W["numin"], W["dnu"], nx, irange=(ib, ie))
    return out


def cpu_baseline(W, L, T, P, seconds, seed=0, max_tiles=None):
    """The FP64 oracle (OpenMP, all host threads) on a bounded sample of grid
    tiles of the same workload.  Returns (summary, {tile: oracle K}): pairs/s,
    what was sampled, and the state's total pairs with the full step time
    they extrapolate to at that rate.  For lists measured on a head of the
    list the tiles' K covers only that head and is not returned."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    head = ""
    if W["n"] > 20_000_000:
        # per-line oracle arrays of a 5e8-line list do not fit the host: the
        # rate is measured on a 2e7-line head of the list (same distributions)
        L = {k: v[:20_000_000] for k, v in L.items()}
        head = ", 2e7-line head of the list"
    nu, S, iad, vy, win, nx = oracle_state(W, L, T, P)
    total = int(np.sum(win[:, 5] - win[:, 0]))
    order = tile_order(nx, seed)
    pairs, tsum, used, Ktiles = 0, 0.0, 0, {}
    for t in order:
        ib, ie = int(t * TILE), int(min(nx, (t + 1) * TILE))
        t0 = time.perf_counter()
        Kt, pr = oracle.opacity(nu, S, iad, vy, win, W["numin"], W["dnu"], nx, irange=(ib, ie))
        tsum += time.perf_counter() - t0
        pairs += sum(pr)
        Ktiles[t] = Kt
        used += 1
        if tsum >= seconds or (max_tiles and used >= max_tiles):
            break
    cores = os.cpu_count() or 1
    rate = pairs / tsum
    if head:
        Ktiles = {}
        total = int(total * (W["n"] / 20_000_000))  # the whole list's pairs, scaled from the head
    return ({"value": rate, "unit": "Voigt evals/s", "cores": cores, "kind": "port",
             "sample": f"{used} random {TILE}-point grid tiles of {len(order)} "
                       f"({pairs:.3e} pairs, {tsum:.1f} s){head}, FP64 oracle, OpenMP {cores} threads",
             "state_pairs": total, "state_s_extrapolated": total / rate},
            Ktiles)


def parity_figure(Kg_tiles, binmax_tiles, Ko_tiles, tol=1e-5):
    """Max relative error of the GPU's K against the oracle's on sampled
    tiles, where K > 1e-6 of its bin maximum (the bin maximum of the GPU's K:
    the oracle sums only the sampled tiles)."""
    worst, pts, used = 0.0, 0, 0
    for t, Ko in Ko_tiles.items():
        if t not in Kg_tiles:
            continue
        Kg, bm = Kg_tiles[t], binmax_tiles[t]
        m = Kg > 1e-6 * bm
        if m.any():
            worst = max(worst, float(np.max(np.abs(Kg[m] - Ko[m]) / np.abs(Ko[m]))))
        pts += int(m.sum())
        used += 1
    return {"max_rel_err": worst, "points": pts, "tiles": used, "tolerance": tol,
            "pass": bool(worst < tol), "oracle": "FP64 CPU restatement",
            "mask": "K > 1e-6 of its bin maximum"}


def gpu_tiles(Krow, tiles, nxb):
    """{tile: (K of the tile, per-point bin maximum)} from one state's K row
    (a torch tensor on the device)."""
    import torch
    nx = Krow.shape[0]
    bmax = Krow[: (nx // nxb) * nxb].view(-1, nxb).max(dim=1).values
    out_k, out_b = {}, {}
    for t in tiles:
        ib, ie = t * TILE, min(nx, (t + 1) * TILE)
        out_k[t] = Krow[ib:ie].double().cpu().numpy()
        bins = torch.arange(ib, ie, device=Krow.device) // nxb
        out_b[t] = bmax[bins].cpu().numpy()
    return out_k, out_b


def run_reference(args):
    """--impl reference: the reference has no CPU path of its own, so the
    reference arm is the FP64 CPU restatement (oracle) on the box's host
    cores, each step a bounded sample of the same workload.  ms_per_step is
    the time of one whole step at the measured rate (the state's pairs /
    pairs per second); sample_s is the wall time of the sample itself."""
    ws, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    W = workload(args.workload)
    L = make_lines(W)
    T, P = W["T"][0], W["P"][0]
    # each step a bounded sample: the whole run stays near a minute
    per_step = max(0.5, min(args.cpu_seconds, 60.0 / max(1, args.steps + args.warmup)))
    vals, secs, cb = [], [], None
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cb, _ = cpu_baseline(W, L, T, P, per_step, seed=k)
        if k >= args.warmup:
            vals.append(cb["value"])
            secs.append(time.perf_counter() - t0)
    v = float(np.mean(vals))
    cb["value"] = v
    cb["state_s_extrapolated"] = cb["state_pairs"] / v
    out = {"impl": "reference", "metric": "Voigt evals/s", "value": v, "unit": "Voigt evals/s",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1e3 * cb["state_pairs"] / v, "ms_per_step_kind":
               "extrapolated: the state's pairs / the sampled pairs per second",
           "sample_s": float(np.mean(secs)), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded; the benchmark configurations' line distributions)",
           "config": workload_config(W),
           "cpu_baseline": cb,
           "e2e": {"value": v, "unit": "Voigt evals/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_adjoint(args):
    """Adjoint workload: one step = forward K(T, P), the seed u = w / K of
    Loss = sum_i w_i log K_i, and the vector-Jacobian product (dLoss/dT,
    dLoss/dP, per-line dLoss/dlog S and dLoss/dgammaL).  1 GPU."""
    import torch
    import hkb
    W = workload("adjoint")
    L = make_lines(W)
    ctx = open_ctx(W, L, 0)
    ctx._numin, ctx._dnu = W["numin"], W["dnu"]
    T, P = W["T"][0], W["P"][0]
    prec = hkb.MIXED if args.precision == "mixed" else hkb.PLAIN_FP64
    nx, n = ctx.nx, ctx.num_lines
    pa, pb, pc = count_pairs(ctx, T, P)
    pairs = pa + pb + pc
    w = torch.as_tensor(np.random.default_rng(7).standard_normal(nx), device="cuda")
    K = torch.empty((1, nx), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        ctx.opacity([T], [P], prec, out=K, stream=stream)
        u = w / K[0]
        return ctx.opacity_vjp(T, P, u, prec)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clk = Clocks(0)
    clk.start()
    t0 = time.perf_counter()
    fwd, vjp = [], []
    for _ in range(args.steps):
        ctx.opacity([T], [P], prec, out=K, stream=stream)
        torch.cuda.synchronize()
        fwd.append(ctx.last_timing()[0])
        ctx.opacity_vjp(T, P, w / K[0], prec)
        vjp.append(ctx.last_timing()[0])
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / args.steps
    clocks = clk.stop()
    fwd_ms = float(np.mean(fwd))
    out = {"metric": "Voigt evals/s (forward + adjoint)", "value": 2 * pairs / (ms * 1e-3),
           "unit": "Voigt evals/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32 profile and derivatives, f64 offsets/strengths/sums" if prec == hkb.MIXED else "f64",
           "data": "synthetic (seeded; the benchmark configurations' line distributions)",
           "config": {"workload": W["label"], "lines": W["n"], "grid_points": nx, "T": T, "P": P,
                      "cut_cm-1": W["cut"], "precision": args.precision,
                      "loss": "sum_i w_i log K_i, w ~ N(0,1)",
                      "timing": "wall clock around synchronous steps"},
           "pairs": {"A": pa, "B": pb, "C": pc}, "forward_voigt_ms": fwd_ms,
           "adjoint_ms": ms - fwd_ms, "adjoint_kernels_ms": float(np.mean(vjp)),
           "adjoint_pairs_per_s": pairs / (float(np.mean(vjp)) * 1e-3), "clocks": clocks,
           # prep 2 + voigt, then prep 2 + the adjoint tile (+ mixed region C) and line kernels
           "gpu_launches": args.steps * (8 if prec == hkb.MIXED else 7)}
    print(json.dumps(out), flush=True)
    ctx.close()


def reference_cuda(W, L, T, P, tunings=(1, 0)):
    """The reference's own CUDA build (oracle/_ref/heliosk: the reference
    sources compiled for sm_100a by oracle/Makefile) beside this library's
    drop-in executable, on one run directory of this workload: K(x) seconds
    as each writes it to Info_<name>.dat (the reference's includes its kernel
    self-tuning when doTuning = 1, so both settings are run).  P may be a list
    (one process over a PFile of pressures, as the reference runs tables)."""
    import shutil
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_run as R
    if not os.path.exists(R.REF_EXE):
        return {"unavailable": "oracle/_ref/heliosk not built (needs the reference sources)"}
    base = tempfile.mkdtemp(prefix="hk_ref_")
    out = {"lines": W["n"], "T": T, "P": P, "note": "K(x) of one state: line sum onto the grid"}
    try:
        data = os.path.join(base, "data")
        R.write_data(data, L)
        runs = [("reference_tuned" if t else "reference_untuned", R.REF_EXE, t) for t in tunings]
        for tag, exe, tune in runs + [("dropin", R.OUR_EXE, 1)]:
            d = os.path.join(base, tag)
            R.write_run(d, data, T, P, W["numin"], W["numax"], W["dnu"], W["cut"], W["nbins"],
                        W["nC"], store_k=0, resample=1, tuning=tune)
            r = R.run(exe, d, timeout=900)
            out[tag] = {"rc": r["rc"], "kx_s": r["info"].get("K(x)"), "lines_s": r["info"].get("Lines"),
                        "input_s": r["info"].get("input"), "wall_s": r["wall_s"]}
        ref = [out[t]["kx_s"] for t in ("reference_tuned", "reference_untuned")
               if t in out and out[t]["rc"] == 0 and out[t]["kx_s"]]
        if ref and out["dropin"]["rc"] == 0 and out["dropin"]["kx_s"]:
            out["kx_speedup_vs_best_reference"] = min(ref) / out["dropin"]["kx_s"]
    except Exception as e:  # a failed run is reported, not fatal
        out["error"] = repr(e)[:300]
    finally:
        shutil.rmtree(base, ignore_errors=True)
    return out


def flop_model(pa, pb, pc, n_iter):
    """Algorithmic FP32 flops of one state from its pairs by region."""
    return pa * F_A + pb * F_B + pc * (F_C0 + F_C_ITER * n_iter)


def n_iter_of(ctx, W, L, T, P, lrank):
    """n_iter of the flop model, from the lines themselves or, for lists too
    large to download per line, from a 2e6-line head of the same list."""
    if ctx.num_lines <= 20_000_000:
        return c_series_iterations(ctx, float(T), float(P))
    Wp = dict(W, n=2_000_000)
    Lp = {k: v[:2_000_000] for k, v in L.items()}
    pctx = open_ctx(Wp, Lp, lrank)
    pctx._numin, pctx._dnu = W["numin"], W["dnu"]
    n = c_series_iterations(pctx, float(T), float(P))
    pctx.close()
    return n


def table_leg(ctx, W, L, args, ws, rank, lrank, stream, fp32_peak):
    """The 600-state T-P table of the same line list (20 T x 30 P): the line
    scaling, Voigt sums and k-distribution fits of every state recorded as
    one CUDA graph (hk_table_build) and replayed (hk_table_run), 1 untimed +
    args.table_steps timed replays.  N ranks split the states (rank r takes
    r, r + N, ...).  Adds the plain-FP64 form on 20 states spread over the
    table, the error against the FP64 oracle on sampled tiles of two states,
    and (rank 0, 1 GPU) the reference's own CUDA build on one temperature
    row of 30 pressures."""
    import torch
    import hkb
    from hkb import synth
    Ta, Pa = synth.table_states()
    mine = rank_states(len(Ta), ws, rank)
    T, P = Ta[mine], Pa[mine]
    ns, nx, nb, nC = len(T), ctx.nx, W["nbins"], W["nC"]
    K = torch.empty((ns, nx), dtype=torch.float64, device="cuda")
    coeff = torch.empty((ns, nb, nC), dtype=torch.float64, device="cuda")
    nxmin = torch.empty((ns, nb), dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    ctx.set_table_mode(0)  # per-batch launches first; mode 1 below
    ctx.table_build(T, P, K, coeff, nxmin, nC=nC, precision=hkb.MIXED)
    build_s = time.perf_counter() - t0
    kernels = ctx.table_kernels
    shape_used, shape_tuned, probe_ms = ctx.tuning_result()
    ctx.table_run(stream)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clk = Clocks(lrank)
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.table_steps):
        ctx.table_run(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ctx.table_status(stream)  # raises if a bounded wait inside the run ran out
    s_table = barrier_max(ws, e0.elapsed_time(e1) / args.table_steps * 1e-3)
    ctx.table_free()
    # the same table as one persistent launch for every state's line prep
    # and sums (table mode 1; same bits), one timed replay after the build
    fused = None
    if not args.no_fused:
        ctx.set_table_mode(1)
        Kf = torch.empty((ns, nx), dtype=torch.float64, device="cuda")
        ctx.table_build(T, P, Kf, coeff, nxmin, nC=nC, precision=hkb.MIXED)
        fk = ctx.table_kernels
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        e0.record(stream)
        ctx.table_run(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.table_status(stream)
        fs = barrier_max(ws, e0.elapsed_time(e1) * 1e-3)
        same = bool(torch.equal(Kf[:: max(1, ns // 8)], K[:: max(1, ns // 8)]))
        ctx.table_free()
        ctx.set_table_mode(0)
        del Kf
        torch.cuda.empty_cache()
        fused = {"s_per_table": fs, "graph_kernels": fk, "replays_timed": 1,
                 "K_equal_to_per_batch_graph": same,
                 "note": "one persistent launch: line prep of state s beside the sums of state s-1"}
    # the timed output of two states on the tiles the oracle samples (before
    # the plain-form leg below overwrites the first rows of K)
    par_states = sorted({0, ns // 2})
    par_tiles = {s: tile_order(nx, 100 + s)[:1] for s in par_states}
    par_gpu = {s: gpu_tiles(K[s], par_tiles[s], nx // nb) for s in par_states}
    # exact pairs of every state (outside the timed region)
    pairs = np.array([ctx.count_pairs(float(T[s]), float(P[s])) for s in range(ns)], np.float64)
    pairs_all = barrier_sum(ws, float(pairs.sum()))
    # flop model: n_iter from four states spread over the table
    probe = np.linspace(0, ns - 1, min(ns, 4)).astype(int)
    n_iter = float(np.mean([n_iter_of(ctx, W, L, T[s], P[s], lrank) if pairs[s, 2] > 0 else 0.0
                            for s in probe]))
    flops = barrier_sum(ws, float(sum(flop_model(*pairs[s], n_iter) for s in range(ns))))
    out = {"workload": "tp-table-1e7-lines-600-states", "states": int(len(Ta)),
           "states_this_rank": int(ns), "T": f"{Ta.min():g}-{Ta.max():g} K x 20",
           "P": f"{Pa.min():.3g}-{Pa.max():.3g} atm x 30 (log)",
           "s_per_table": s_table, "replays_timed": args.table_steps,
           "execution": "per-batch line prep + persistent Voigt launches, one k-distribution launch",
           "fused_single_launch": fused,
           "value": pairs_all / s_table, "unit": "Voigt evals/s",
           "pairs": pairs_all, "build_s": build_s, "graph_kernels": kernels,
           "tile_shape": {"shape": shape_used, "tuned": shape_tuned >= 0,
                          "probe_ms": [round(float(v), 3) for v in probe_ms]
                          if shape_tuned >= 0 else None},
           "roofline": {"bound": "fp32", "kernel": "whole replay (line prep, Voigt sums, fits)",
                        "achieved": flops / s_table / 1e12 / ws, "peak": fp32_peak,
                        "unit": "TFLOP/s", "frac": flops / s_table / 1e12 / ws / fp32_peak,
                        "C_series_iters": n_iter},
           "clocks": clocks}
    # error against the FP64 oracle: one sampled tile of two states
    if rank == 0 and not args.no_cpu_baseline:
        par = []
        for s in par_states:
            kg, bm = par_gpu[s]
            _, ko = cpu_baseline(W, L, float(T[s]), float(P[s]), 1e9, seed=100 + s, max_tiles=1)
            par.append(parity_figure(kg, bm, ko))
        out["parity"] = {"max_rel_err": max(p["max_rel_err"] for p in par),
                         "points": sum(p["points"] for p in par),
                         "tiles": sum(p["tiles"] for p in par),
                         "states": [int(mine[s]) for s in par_states],
                         "tolerance": 1e-5, "pass": all(p["pass"] for p in par),
                         "oracle": "FP64 CPU restatement", "mask": par[0]["mask"]}
    # plain FP64 form against the mixed form on 20 states spread over the table
    if not args.no_plain:
        sub = np.linspace(0, ns - 1, min(ns, 20)).astype(int)
        Ks = K[: len(sub)]

        def sub_ms(pr):
            ctx.opacity(T[sub], P[sub], pr, out=Ks, stream=stream)
            ctx.kdist(Ks, nC=nC, stream=stream)
            torch.cuda.synchronize()
            e0.record(stream)
            ctx.opacity(T[sub], P[sub], pr, out=Ks, stream=stream)
            ctx.kdist(Ks, nC=nC, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            return barrier_max(ws, e0.elapsed_time(e1))
        mms, pms = sub_ms(hkb.MIXED), sub_ms(hkb.PLAIN_FP64)
        out["plain_fp64"] = {"subset_states": len(sub), "mixed_ms": mms, "plain_ms": pms,
                             "speedup_mixed_vs_plain": pms / mms,
                             "plain_s_per_table_est": pms * 1e-3 * len(Ta) / len(sub) / ws}
    if rank == 0 and ws == 1 and not args.no_reference_cuda:
        # the reference runs a table as one process per T over a PFile of the
        # 30 pressures: the middle temperature is run, x20 extrapolates
        Tm = float(np.unique(Ta)[len(np.unique(Ta)) // 2])
        Pt = [float(p) for t, p in zip(Ta, Pa) if t == Tm]
        rc = reference_cuda(W, L, Tm, Pt, tunings=(1,))
        nT = len(np.unique(Ta))
        rc["table_extrapolation"] = f"one T ({Tm:.6g} K) x {len(Pt)} P run; x{nT} for the table"
        for t in ("reference_tuned", "dropin"):
            if t in rc and rc[t].get("kx_s"):
                rc[t]["kx_s_table_est"] = rc[t]["kx_s"] * nT
        if rc.get("reference_tuned", {}).get("kx_s"):
            rc["table_speedup_vs_reference_kx"] = rc["reference_tuned"]["kx_s"] * nT / s_table
        out["reference_cuda"] = rc
    del K, coeff, nxmin
    torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "adjoint":
        run_adjoint(args)
        return
    ws, rank, lrank = dist_setup(args)
    import torch
    import hkb
    torch.cuda.set_device(lrank)
    W = workload(args.workload)
    L = make_lines(W)
    ctx = open_ctx(W, L, lrank)
    ctx._numin, ctx._dnu = W["numin"], W["dnu"]
    T = np.array(W["T"], np.float64)
    P = np.array(W["P"], np.float64)
    if args.workload == "table" and ws > 1:
        # the table workload on N ranks: disjoint states per rank
        mine = rank_states(len(T), ws, rank)
        T, P = T[mine], P[mine]
    ns, nx, nb, nC = len(T), ctx.nx, W["nbins"], W["nC"]
    prec = hkb.MIXED if args.precision == "mixed" else hkb.PLAIN_FP64

    # exact algorithmic work (outside the timed region)
    per_state = [count_pairs(ctx, float(T[s]), float(P[s])) for s in range(ns)]
    pa, pb, pc = (float(np.mean([p[k] for p in per_state])) for k in range(3))
    pairs_step = (pa + pb + pc) * ns
    n_iter = n_iter_of(ctx, W, L, T[0], P[0], lrank) if pc > 0 else 0.0
    flops_step = ns * flop_model(pa, pb, pc, n_iter)

    stream = torch.cuda.current_stream()
    K = torch.empty((ns, nx), dtype=torch.float64, device="cuda")
    coeff = torch.empty((ns, nb, nC), dtype=torch.float64, device="cuda")
    nxmin = torch.empty((ns, nb), dtype=torch.int32, device="cuda")

    def step(precision):
        ctx.opacity(T, P, precision, out=K, stream=stream)
        ctx.kdist(K, nC=nC, stream=stream)

    # one step = the whole batch of states (line prep, Voigt sums, fits)
    # replayed as one CUDA graph (hk_table_build / hk_table_run); line lists
    # whose per-state records exceed the workspace run the sectioned path of
    # hk_opacity instead (not capturable: it sizes sections from the state
    # pass)
    # the tile shape is tuned once, before the graph is recorded (outside
    # the timed steps, like the workspace allocations)
    ctx.set_tuning(args.tuning)
    ctx.set_table_mode(args.table_mode)
    try:
        ctx.table_build(T, P, K, coeff, nxmin, nC=nC, precision=prec)
        graph = True
    except hkb.HkError as err:
        if err.status != -8:  # HK_ERR_UNSUPPORTED
            raise
        graph = False

    def timed_step():
        if graph:
            ctx.table_run(stream)
        else:
            step(prec)

    for _ in range(args.warmup):
        timed_step()
    torch.cuda.synchronize()
    launches_per_step = ctx.table_kernels if graph else ctx.last_launches
    shape_used, shape_tuned, probe_ms = ctx.tuning_result()
    if ws > 1:
        torch.distributed.barrier()
    clk = Clocks(lrank)
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        timed_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    clocks = clk.stop()
    if graph:
        ctx.table_status(stream)  # raises if a bounded wait inside a run ran out
    ms = barrier_max(ws, ms)
    # the timed output on the tiles the oracle samples (before anything else
    # overwrites K)
    nxb = nx // nb
    sample = tile_order(nx, 0)[:32]
    Kg_tiles, bmax_tiles = gpu_tiles(K[0], sample, nxb)
    if graph:
        ctx.table_free()

    # dominant kernel: per-launch device time with CUDA events on the stream
    vms, kms = [], []
    for _ in range(max(3, min(args.steps, 10))):
        step(prec)
        v, k = ctx.last_timing()
        vms.append(v)
        kms.append(k)
    voigt_ms = float(np.mean(vms))
    kdist_ms = float(np.mean(kms))
    fp32_peak = ctx.fp32_peak_tflops()

    # end to end through the public API with host buffers: states in, the
    # k-distribution fit out to host memory, and for a single state K too
    # (a T-P table's product is its fit: its K stays on the device)
    K_host = torch.empty((ns, nx), dtype=torch.float64, pin_memory=True) if ns == 1 else None
    # K's copy to the host runs on its own stream beside the fit (both only
    # read K)
    copy_stream = torch.cuda.Stream()
    k_done = torch.cuda.Event()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.opacity(T, P, prec, out=K, stream=stream)
        if K_host is not None:
            k_done.record(stream)
            copy_stream.wait_event(k_done)
            with torch.cuda.stream(copy_stream):
                K_host.copy_(K, non_blocking=True)
        r = ctx.kdist(K, nC=nC, stream=stream, outputs_on_device=False)
        torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / args.steps
    e2e_s = barrier_max(ws, e2e_s)
    d2h = ns * nb * (nC * 8 + 4) + (ns * nx * 8 if ns == 1 else 0)

    plain = None
    if not args.no_plain and args.precision == "mixed" and ns == 1:
        for _ in range(1):
            step(hkb.PLAIN_FP64)
        torch.cuda.synchronize()
        e0.record(stream)
        nplain = max(1, min(3, args.steps))
        for _ in range(nplain):
            step(hkb.PLAIN_FP64)
        e1.record(stream)
        torch.cuda.synchronize()
        pms = barrier_max(ws, e0.elapsed_time(e1) / nplain)
        plain = {"ms_per_step": pms, "value": pairs_step * ws / (pms * 1e-3),
                 "speedup_mixed_vs_plain": pms / ms}
    elif not args.no_plain and args.precision == "mixed":
        # a table's plain FP64 run takes minutes: both forms on the same
        # states spread over the table (20 of a T-P table, 1 of a 5e8-line
        # list), opacity + fit, 1 untimed + 1 timed
        nsub = 1 if W.get("database") == "exomol" else 20
        sub = np.linspace(0, ns - 1, min(ns, nsub)).astype(int)
        Ks = K[:len(sub)]

        def sub_ms(pr):
            ctx.opacity(T[sub], P[sub], pr, out=Ks, stream=stream)
            ctx.kdist(Ks, nC=nC, stream=stream)
            torch.cuda.synchronize()
            e0.record(stream)
            ctx.opacity(T[sub], P[sub], pr, out=Ks, stream=stream)
            ctx.kdist(Ks, nC=nC, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            return barrier_max(ws, e0.elapsed_time(e1))

        mms, pms = sub_ms(hkb.MIXED), sub_ms(hkb.PLAIN_FP64)
        plain = {"subset_states": len(sub), "mixed_ms": mms, "plain_ms": pms,
                 "speedup_mixed_vs_plain": pms / mms,
                 "plain_s_per_table_est": pms * 1e-3 * ns / len(sub)}

    value = pairs_step * ws / (ms * 1e-3)
    out = {
        "metric": "Voigt evals/s", "value": value, "unit": "Voigt evals/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 profile, f64 offsets/strengths/sum/fit" if prec == hkb.MIXED else "f64",
        "data": "synthetic (seeded; the benchmark configurations' line distributions)",
        "config": workload_config(W),
        "precision": args.precision,
        "parallelism": f"{'states split' if args.workload == 'table' and ws > 1 else 'replicas'} "
                       f"x{ws} ranks",
        "execution": {"mode": "one CUDA graph per step" if graph else "hk_opacity sections + hk_kdist",
                      "tile_shape": {"lines_per_chunk": hkb.tile_shape(shape_used)[0],
                                     "points_per_tile": hkb.tile_shape(shape_used)[1],
                                     "warps": hkb.tile_shape(shape_used, warps=True)[2],
                                     "shape": shape_used, "tuned": shape_tuned >= 0,
                                     "probe_ms": [round(float(v), 3) for v in probe_ms]
                                     if shape_tuned >= 0 else None}},
        "s_per_state": ms * 1e-3 / ns,
        "s_per_table": ms * 1e-3 if ns > 1 else None,
        "pairs_per_state": {"A": pa, "B": pb, "C": pc, "C_series_iters": n_iter},
        "roofline": {"bound": "fp32", "kernel": "voigt_sum_kernel",
                     "achieved": flops_step / (voigt_ms * 1e-3) / 1e12,
                     "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": flops_step / (voigt_ms * 1e-3) / 1e12 / fp32_peak,
                     "traffic": VOIGT_DRAM_BYTES.get(W["label"]) if prec == hkb.MIXED else None,
                     "voigt_ms": voigt_ms, "kdist_ms": kdist_ms,
                     "peak_source": "in-run FP32 FMA probe (hk_fp32_peak); "
                                    "MEASURED_PEAKS.json has no FP32 SIMT figure"},
        "e2e": {"value": pairs_step * ws / e2e_s, "unit": "Voigt evals/s",
                "h2d_bytes_per_step": SIZEOF_STATE * ns,
                "d2h_bytes_per_step": d2h},
        "clocks": clocks,
        "gpu_launches": launches_per_step * args.steps,
        "plain_fp64": plain,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cb, Ko = cpu_baseline(W, L, float(T[0]), float(P[0]), args.cpu_seconds,
                              max_tiles=len(sample))
        if not Ko:
            # a head-of-list rate sample: the tiles' oracle K from every line
            # that can reach them instead
            Ko = oracle_tiles_near(W, L, float(T[0]), float(P[0]), sample[:2])
        out["cpu_baseline"] = cb
        out["parity"] = parity_figure(Kg_tiles, bmax_tiles, Ko,
                                      tol=1e-5 if prec == hkb.MIXED else 1e-12)
    if rank == 0 and ws == 1 and ns == 1 and not args.no_reference_cuda:
        out["reference_cuda"] = reference_cuda(W, L, float(T[0]), float(P[0]))
    elif rank == 0 and ws == 1 and args.workload == "table" and not args.no_reference_cuda:
        # the reference runs a table as one process per T over a PFile of the
        # 30 pressures: the middle temperature is run, x20 extrapolates
        Tm = sorted(set(W["T"]))[len(set(W["T"])) // 2]
        Pt = [p for t, p in zip(W["T"], W["P"]) if t == Tm]
        rc = reference_cuda(W, L, Tm, Pt, tunings=(1,))
        nT = len(set(W["T"]))
        rc["table_extrapolation"] = f"one T ({Tm:.6g} K) x {len(Pt)} P run; x{nT} for the table"
        for t in ("reference_tuned", "dropin"):
            if t in rc and rc[t].get("kx_s"):
                rc[t]["kx_s_table_est"] = rc[t]["kx_s"] * nT
        out["reference_cuda"] = rc
    if args.workload == "hitemp" and prec == hkb.MIXED and not args.no_table:
        del K, coeff, nxmin
        torch.cuda.empty_cache()
        tab = table_leg(ctx, W, L, args, ws, rank, lrank, stream, fp32_peak)
        out["table"] = tab
        out["s_per_table"] = tab["s_per_table"]
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
