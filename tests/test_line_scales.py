"""GPU: per-line multipliers of S and gammaL set from device arrays
(hk_set_line_scales_device) against the host entry point (hk_set_line_scales).

The two routes must give the same K to the bit, in both precisions, since
they place the same values in the same sorted order.  A value that is not
finite and > 0 is refused with its load index and leaves no multiplier in
force; a pointer that is not device memory of the context's GPU is refused
before anything runs.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import hkb
from hkb import synth

pytestmark = pytest.mark.gpu

NUMIN, NUMAX, DNU, NBINS = 1000.0, 1300.0, 0.01, 10
T0, P0 = 800.3, 1.0


@pytest.fixture(scope="module")
def scl():
    L = synth.hitran_lines(800, seed=5, nu_max=NUMAX, nu_min=NUMIN)
    Tq, Qq = synth.q_table()
    ctx = hkb.Context(0)
    ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
    ctx.set_partition(0, Tq, Qq)
    ctx.set_options(qalphaL=1.0)
    ctx.load_lines_hitran(L)
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    rng = np.random.default_rng(3)
    n = ctx.num_lines
    s = np.exp(rng.normal(0.0, 0.5, n))
    g = np.exp(rng.normal(0.0, 0.3, n))
    yield dict(ctx=ctx, s=s, g=g)
    ctx.close()


@pytest.mark.parametrize("prec", [hkb.MIXED, hkb.PLAIN_FP64])
def test_device_scales_equal_host_scales(scl, prec):
    ctx, s, g = scl["ctx"], scl["s"], scl["g"]
    ctx.set_line_scales(s, g)
    Kh = ctx.opacity([T0], [P0], prec)[0]
    ctx.set_line_scales(torch.as_tensor(s, device="cuda"), torch.as_tensor(g, device="cuda"))
    Kd = ctx.opacity([T0], [P0], prec)[0]
    ctx.set_line_scales(None, None)
    K1 = ctx.opacity([T0], [P0], prec)[0]
    assert np.array_equal(Kh, Kd)
    assert not np.array_equal(Kd, K1)  # the multipliers took effect
    # one of the two, the other restored to 1
    ctx.set_line_scales(torch.as_tensor(s, device="cuda"), None)
    Kd = ctx.opacity([T0], [P0], prec)[0]
    ctx.set_line_scales(s, None)
    Kh = ctx.opacity([T0], [P0], prec)[0]
    ctx.set_line_scales()
    assert np.array_equal(Kh, Kd)


def test_device_scales_invalid_value(scl):
    ctx, s, g = scl["ctx"], scl["s"], scl["g"]
    K1 = ctx.opacity([T0], [P0], hkb.MIXED)[0]
    bad = s.copy()
    bad[[17, 400]] = [np.nan, -1.0]
    ctx.set_line_scales(torch.as_tensor(s, device="cuda"), torch.as_tensor(g, device="cuda"))
    with pytest.raises(hkb.HkError, match="line scale 17 "):
        ctx.set_line_scales(torch.as_tensor(s, device="cuda"), torch.as_tensor(bad, device="cuda"))
    # refused: neither multiplier stays in force
    assert np.array_equal(ctx.opacity([T0], [P0], hkb.MIXED)[0], K1)
    inf = g.copy()
    inf[5] = np.inf
    with pytest.raises(hkb.HkError, match="line scale 5 "):
        ctx.set_line_scales(torch.as_tensor(inf, device="cuda"), None)
    assert np.array_equal(ctx.opacity([T0], [P0], hkb.MIXED)[0], K1)


def test_device_scales_refuse_host_memory(scl):
    ctx, s = scl["ctx"], scl["s"]
    st = hkb.lib().hk_set_line_scales_device(ctx._h, s.ctypes.data_as(C.c_void_p), None, None)
    assert hkb.STATUS_NAMES[st] == "HK_ERR_ARG"
    ctx.set_line_scales()


def test_autograd_device_scales(scl):
    """The autograd bridge keeps log S and log gammaL on the GPU; its
    forward equals the host route's K."""
    from hkb.autograd import Opacity
    ctx, s, g = scl["ctx"], scl["s"], scl["g"]
    ls = torch.as_tensor(np.log(s), device="cuda").requires_grad_(True)
    lg = torch.as_tensor(np.log(g), device="cuda").requires_grad_(True)
    K = Opacity.apply(ctx, T0, P0, ls, lg, hkb.PLAIN_FP64)
    ctx.set_line_scales(torch.exp(ls).detach().cpu().numpy(), torch.exp(lg).detach().cpu().numpy())
    Kh = ctx.opacity([T0], [P0], hkb.PLAIN_FP64)[0]
    ctx.set_line_scales()
    assert np.array_equal(K.detach().cpu().numpy(), Kh)
    K.log().sum().backward()
    assert ls.grad is not None and lg.grad is not None
    assert torch.isfinite(ls.grad).all() and torch.isfinite(lg.grad).all()
