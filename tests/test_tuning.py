"""GPU: tile shapes of the mixed Voigt kernel and the shape autotuner.

Every shape (lines per staged chunk x grid points per tile) must meet the
mixed-form bound against the FP64 oracle (1e-5 relative where K > 1e-6 of
its bin maximum) and keep the per-shape invariants of the default one:
batching and grid sections do not change a bit of K.  The tuner's choice is
one of the shapes, is what the following calls run, and is dropped when the
grid changes.
"""
import numpy as np
import pytest

import hkb
from hkb import synth
from test_gpu_parity import NBINS, DNU, NUMAX, NUMIN, STATES, masked_relerr, oracle_state

pytestmark = pytest.mark.gpu

NSHAPES = 7


@pytest.fixture(scope="module")
def small():
    L = synth.hitran_lines(20000, seed=11, nu_max=3000.0)
    Tq, Qq = synth.q_table()
    ctx = hkb.Context(0)
    ctx.set_species(hkb.HITRAN, [synth.MASS], [1.0])
    ctx.set_partition(0, Tq, Qq)
    ctx.set_options(qalphaL=1.0)
    ctx.load_lines_hitran(L)
    yield dict(ctx=ctx, L=L, Tq=Tq, Qq=Qq)
    ctx.close()


def test_shape_table():
    assert hkb.num_tile_shapes() == NSHAPES
    shapes = [hkb.tile_shape(v, warps=True) for v in range(NSHAPES)]
    assert shapes[0] == (128, 2048, 8) and hkb.tile_points() == 2048
    assert len(set(shapes)) == NSHAPES
    for ch, g, w in shapes:
        assert ch % 32 == 0 and 2048 % g == 0 and ch <= 32 * w
    with pytest.raises(hkb.HkError):
        hkb.tile_shape(NSHAPES)


@pytest.mark.parametrize("shape", range(NSHAPES))
def test_each_shape_matches_oracle(small, shape):
    ctx = small["ctx"]
    ctx.set_tuning(0)
    ctx.set_tile_shape(shape)
    try:
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        Ts = np.array([s[0] for s in STATES])
        Ps = np.array([s[1] for s in STATES])
        Kb = ctx.opacity(Ts, Ps, hkb.MIXED)
        assert ctx.tuning_result()[0] == shape
        for s, (T, P) in enumerate(STATES):
            Kref, _, _ = oracle_state(small, T, P)
            err, _ = masked_relerr(Kb[s], Kref, NBINS)
            print(f"shape {shape} {hkb.tile_shape(shape)} T={T} P={P} mixed {err:.2e}")
            assert err < 1e-5
            assert np.array_equal(ctx.opacity([T], [P], hkb.MIXED)[0], Kb[s])
        # the plain FP64 form keeps the default shape whatever is set
        ctx.opacity([1000.0], [1.0], hkb.PLAIN_FP64)
    finally:
        ctx.set_tile_shape(0)


def test_sections_bit_identical_for_a_narrow_shape(small):
    ctx = small["ctx"]
    ctx.set_tuning(0)
    ctx.set_tile_shape(3)
    try:
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        Ts, Ps = np.array([1500.0, 300.0]), np.array([0.1, 10.0])
        ref = ctx.opacity(Ts, Ps, hkb.MIXED)
        ctx.set_workspace(prep_bytes=3000 * 112, part_bytes=4 * 2**30)
        assert np.array_equal(ctx.opacity(Ts, Ps, hkb.MIXED), ref)
    finally:
        ctx.set_workspace()
        ctx.set_tile_shape(0)


def test_tuner_choice_runs_and_resets(small):
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    Ts = np.array([300.0, 1000.0, 2500.0, 1500.0])
    Ps = np.array([1e-6, 1.0, 100.0, 0.1])
    try:
        ctx.set_tuning(2)
        Kt = ctx.opacity(Ts, Ps, hkb.MIXED)
        last, tuned, ms = ctx.tuning_result()
        print("probe ms per shape", ms, "->", tuned)
        assert 0 <= tuned < NSHAPES and last == tuned
        assert np.all(ms > 0.0) and ms[tuned] == ms.min()
        # the cached choice serves the next call without new probes
        assert np.array_equal(ctx.opacity(Ts, Ps, hkb.MIXED), Kt)
        ctx.set_tuning(0)
        ctx.set_tile_shape(tuned)
        assert np.array_equal(ctx.opacity(Ts, Ps, hkb.MIXED), Kt)
        ctx.set_tuning(2)
        ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
        assert ctx.tuning_result()[1] == -1  # a new grid drops the choice
    finally:
        ctx.set_tuning(0)
        ctx.set_tile_shape(0)


def test_tuning_mode1_pays_off_only_for_batches(small):
    import torch
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    try:
        ctx.set_tuning(1)
        ctx.opacity([1500.0], [0.1], hkb.MIXED)
        assert ctx.tuning_result()[1] == -1  # probes would cost more than the call
        ns = 40 * NSHAPES + 20  # probes: shapes x 4 states x the whole grid <= 10 % of the call
        T = np.linspace(200.0, 3000.0, ns)
        P = 10.0 ** np.linspace(-6.0, 2.0, ns)
        K = torch.empty((ns, ctx.nx), dtype=torch.float64, device="cuda")
        ctx.opacity(T, P, hkb.MIXED, out=K)
        torch.cuda.synchronize()
        last, tuned, _ = ctx.tuning_result()
        assert 0 <= tuned < NSHAPES and last == tuned
        Kref, _, _ = oracle_state(small, T[37], P[37])
        assert masked_relerr(K[37].cpu().numpy(), Kref, NBINS)[0] < 1e-5
    finally:
        ctx.set_tuning(0)


def test_table_build_tunes_before_recording(small):
    import torch
    ctx = small["ctx"]
    ctx.set_grid(NUMIN, NUMAX, DNU, NBINS, 0, 25.0)
    Ts = np.array([300.0, 1000.0, 2500.0, 700.0, 1500.0, 120.0])
    Ps = np.array([1e-6, 1.0, 100.0, 1e-3, 0.1, 10.0])
    ns, nx, nC = len(Ts), ctx.nx, 20
    K = torch.empty((ns, nx), dtype=torch.float64, device="cuda")
    coeff = torch.empty((ns, NBINS, nC), dtype=torch.float64, device="cuda")
    nxmin = torch.empty((ns, NBINS), dtype=torch.int32, device="cuda")
    try:
        ctx.set_tuning(2)
        ctx.table_build(Ts, Ps, K, coeff, nxmin, nC=nC)
        tuned = ctx.tuning_result()[1]
        assert 0 <= tuned < NSHAPES
        ctx.table_run()
        torch.cuda.synchronize()
        K1 = K.cpu().numpy()
        ctx.table_free()
        ctx.set_tuning(0)
        ctx.set_tile_shape(tuned)
        assert np.array_equal(ctx.opacity(Ts, Ps, hkb.MIXED), K1)
    finally:
        ctx.set_tuning(0)
        ctx.set_tile_shape(0)
