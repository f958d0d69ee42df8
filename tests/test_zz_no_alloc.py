"""hk_kdist_noalloc: the per-bin sort + Chebyshev fit for callers that cannot
allocate device memory (a host program that owns all GPU memory through its
own pool or a fixed budget, or that must not make allocation calls that can
synchronise the device or fail mid-run).  It must agree with hk_kdist, which
keeps its QR workspace in memory the library allocates, on the same K.

Collected last on purpose (file name), so a run that stops at the first
failure has already run every other test.  It also runs alone in a fresh
process: nothing here depends on earlier tests.
"""
import ctypes

import numpy as np
import pytest

import hkb
from hkb import synth

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS, NC = 0.0, 3000.0, 0.01, 30, 20


def _noalloc(K, ns, nx, nbins, nC, kmin, coeff, nxmin, sortedK, stream):
    err = ctypes.create_string_buffer(256)
    st = hkb.lib().hk_kdist_noalloc(
        ctypes.c_void_p(K.data_ptr()), ns, nx, nbins, nC, kmin, 1.0,
        ctypes.c_void_p(coeff.data_ptr()), ctypes.c_void_p(nxmin.data_ptr()),
        ctypes.c_void_p(sortedK.data_ptr()) if sortedK is not None else None,
        ctypes.c_void_p(stream.cuda_stream), err, 256)
    return st, err.value.decode()


def test_kdist_noalloc_matches_kdist_twice():
    import torch
    L = synth.hitran_lines(20000, seed=11, nu_max=3000.0)
    Tq, Qq = synth.q_table()
    with hkb.Context(0) as ctx:
        ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
        ctx.set_partition(0, Tq, Qq)
        ctx.set_options(qalphaL=1.0)
        ctx.load_lines_hitran(L)
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        nx = ctx.nx
        K = torch.empty((2, nx), dtype=torch.float64, device="cuda")
        ctx.opacity([1500.0, 800.0], [0.1, 1.0], hkb.MIXED, out=K)
        # a floor inside the data range exercises the partly-empty-bin rules
        kmin = float(torch.quantile(K[1, : nx // 3].cpu(), 0.4))
        K[1].clamp_(min=kmin)
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0, kmin)
        ref = ctx.kdist(K, nC=NC, sorted_K=True)
        torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    for call in range(2):
        coeff = torch.full((2, NBINS, NC), float("nan"), dtype=torch.float64, device="cuda")
        nxmin = torch.full((2, NBINS), -1, dtype=torch.int32, device="cuda")
        sortedK = torch.full((2, nx), float("nan"), dtype=torch.float64, device="cuda")
        st, msg = _noalloc(K, 2, nx, NBINS, NC, kmin, coeff, nxmin, sortedK, stream)
        assert st == hkb.HK_OK, msg
        torch.cuda.synchronize()
        assert torch.equal(sortedK, ref["sorted"]), f"call {call}: sorted bins differ"
        assert torch.equal(nxmin, ref["nxmin"]), f"call {call}: Nxmin differs"
        ok = (ref["nxmin"] < nx // NBINS).unsqueeze(-1).expand_as(coeff)
        err = (coeff - ref["coeff"]).abs()[ok].max().item()
        assert err < 1e-9, f"call {call}: coefficient max abs difference {err}"


def test_kdist_noalloc_rejects_oversize():
    import torch
    nx = 300000
    K = torch.ones((1, nx), dtype=torch.float64, device="cuda")
    coeff = torch.empty((1, 1, NC), dtype=torch.float64, device="cuda")
    nxmin = torch.empty((1, 1), dtype=torch.int32, device="cuda")
    st, msg = _noalloc(K, 1, nx, 1, NC, 0.0, coeff, nxmin, None, torch.cuda.current_stream())
    assert st == -4, (st, msg)
    assert "fixed scratch" in msg
