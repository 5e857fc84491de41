"""The batched persistent forward against the per-pair forward (bit for bit: the same
per-cell arithmetic, only the work schedule differs) and against the oracle."""
import numpy as np
import pytest
import torch

from conftest import assert_bitexact
from hindemith_b200 import _lib as L
from hindemith_b200 import device as D
from hindemith_b200 import synthetic
from hindemith_b200.autotune import BATCH_CANDIDATES
from hindemith_b200.batched import BatchPlan, forward_batched
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu

MIXED = [(1, 1, 1.0, 3), (7, 130, 0.5, 9), (65, 127, 1.7, 40), (300, 518, 0.8, 37),
         (130, 7, 1.2, 0), (240, 320, 2.0, 100), (480, 640, 0.6, 23), (33, 65, 1.0, 8)]


def make_inputs(specs, seed0=1000):
    out = []
    for i, (H, W, _, _) in enumerate(specs):
        I0, I1, _, _ = synthetic.make_pair(H, W, seed=seed0 + i)
        out.append((I0, I1))
    return out


def run_plan(specs, cfg, inputs):
    plan = BatchPlan(specs, cfg)
    for i, (I0, I1) in enumerate(inputs):
        plan.I0[i].copy_(torch.from_numpy(I0))
        plan.I1[i].copy_(torch.from_numpy(I1))
    plan.run()
    plan.check()
    return plan


@pytest.mark.parametrize("T,fast", [(4, False), (4, True), (3, False), (5, True), (1, False), (8, True)])
def test_batched_equals_per_pair(cuda, T, fast):
    cfg = L.make_config(sweeps_per_pass=T, fast_math=fast)
    inputs = make_inputs(MIXED)
    plan = run_plan(MIXED, cfg, inputs)
    for i, ((H, W, alpha, iters), (I0, I1)) in enumerate(zip(MIXED, inputs)):
        u, v = D.hs_forward(D.as_plane(torch.from_numpy(I0).cuda()),
                            D.as_plane(torch.from_numpy(I1).cuda()), alpha, iters, cfg)
        torch.cuda.synchronize()
        assert_bitexact(plan.u[i].cpu().numpy(), u.cpu().numpy(), f"u pair {i}")
        assert_bitexact(plan.v[i].cpu().numpy(), v.cpu().numpy(), f"v pair {i}")


def test_batched_exact_equals_oracle(cuda):
    specs = [(65, 127, 1.7, 40), (300, 518, 0.8, 37), (1, 9, 1.0, 5)]
    inputs = make_inputs(specs, 2000)
    plan = run_plan(specs, L.make_config(sweeps_per_pass=4), inputs)
    for i, ((H, W, alpha, iters), (I0, I1)) in enumerate(zip(specs, inputs)):
        ru, rv = O.c_hs_forward(I0, I1, np.float32(alpha), iters)
        assert_bitexact(plan.u[i].cpu().numpy(), ru, f"u pair {i}")
        assert_bitexact(plan.v[i].cpu().numpy(), rv, f"v pair {i}")


def test_batched_segment_sizes(cuda):
    """Small segments make many dependent tiles per pass; results must not change."""
    specs = [(200, 300, 1.0, 24), (97, 61, 0.7, 16)]
    inputs = make_inputs(specs, 3000)
    ref = run_plan(specs, L.make_config(sweeps_per_pass=4), inputs)
    for rows in (4, 5, 17):
        plan = run_plan(specs, L.make_config(sweeps_per_pass=4, rows_per_segment=rows), inputs)
        for i in range(len(specs)):
            assert_bitexact(plan.u[i].cpu().numpy(), ref.u[i].cpu().numpy(), f"u rows={rows}")
            assert_bitexact(plan.v[i].cpu().numpy(), ref.v[i].cpu().numpy(), f"v rows={rows}")


def test_batched_graph_capture_and_replay(cuda):
    specs = MIXED[:5]
    inputs = make_inputs(specs, 4000)
    cfg = L.make_config(sweeps_per_pass=4, fast_math=True)
    eager = run_plan(specs, cfg, inputs)
    plan = BatchPlan(specs, cfg)
    for i, (I0, I1) in enumerate(inputs):
        plan.I0[i].copy_(torch.from_numpy(I0))
        plan.I1[i].copy_(torch.from_numpy(I1))
    plan.capture()
    for _ in range(2):
        for t in plan.u + plan.v:
            t.fill_(float("nan"))
        plan.replay()
        torch.cuda.synchronize()
        plan.check()
        for i in range(len(specs)):
            assert_bitexact(plan.u[i].cpu().numpy(), eager.u[i].cpu().numpy(), f"u pair {i}")
            assert_bitexact(plan.v[i].cpu().numpy(), eager.v[i].cpu().numpy(), f"v pair {i}")


def test_forward_batched_eager_api(cuda):
    specs = [(40, 52, 1.0, 12), (17, 9, 0.5, 7)]
    inputs = make_inputs(specs, 5000)
    pairs = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), s[2], s[3])
             for (a, b), s in zip(inputs, specs)]
    outs = forward_batched(pairs, L.make_config(sweeps_per_pass=4))
    torch.cuda.synchronize()
    for (u, v), (a, b), s in zip(outs, inputs, specs):
        ru, rv = O.c_hs_forward(a, b, np.float32(s[2]), s[3])
        assert_bitexact(u.cpu().numpy(), ru, "u")
        assert_bitexact(v.cpu().numpy(), rv, "v")


@pytest.mark.parametrize("T", [3, 4, 6, 8])
def test_batched_wide_layout_equals_per_pair(cuda, T):
    """The persistent launch in the 4-columns-per-lane layout (128-column tiles) equals the
    per-pair forward in the 2-column layout, bit for bit."""
    inputs = make_inputs(MIXED)
    plan = run_plan(MIXED, L.make_config(sweeps_per_pass=T, fast_math=True, layout=2), inputs)
    narrow = L.make_config(sweeps_per_pass=T, fast_math=True, layout=1)
    for i, ((H, W, alpha, iters), (I0, I1)) in enumerate(zip(MIXED, inputs)):
        u, v = D.hs_forward(D.as_plane(torch.from_numpy(I0).cuda()),
                            D.as_plane(torch.from_numpy(I1).cuda()), alpha, iters, narrow)
        torch.cuda.synchronize()
        assert_bitexact(plan.u[i].cpu().numpy(), u.cpu().numpy(), f"u pair {i}")
        assert_bitexact(plan.v[i].cpu().numpy(), v.cpu().numpy(), f"v pair {i}")


@pytest.mark.parametrize("T,rows,layout", BATCH_CANDIDATES)
def test_batched_every_tuner_candidate_equals_per_pair(cuda, T, rows, layout):
    """Each (depth, rows per tile, layout) the batch autotuner may pick, in the fast form
    the benchmark runs: equal to the per-pair forward bit for bit."""
    inputs = make_inputs(MIXED, 6000)
    plan = run_plan(MIXED, L.make_config(sweeps_per_pass=T, rows_per_segment=rows,
                                         fast_math=True, layout=layout), inputs)
    narrow = L.make_config(sweeps_per_pass=T, fast_math=True, layout=1)
    for i, ((H, W, alpha, iters), (I0, I1)) in enumerate(zip(MIXED, inputs)):
        u, v = D.hs_forward(D.as_plane(torch.from_numpy(I0).cuda()),
                            D.as_plane(torch.from_numpy(I1).cuda()), alpha, iters, narrow)
        torch.cuda.synchronize()
        assert_bitexact(plan.u[i].cpu().numpy(), u.cpu().numpy(), f"u pair {i}")
        assert_bitexact(plan.v[i].cpu().numpy(), v.cpu().numpy(), f"v pair {i}")


def test_bounded_wait_times_out_and_context_survives(cuda):
    """A device-side wait on a flag that nothing sets gives up after its poll limit and
    reports HS_ERR_TIMEOUT through the status word; the context stays usable."""
    import ctypes
    import time

    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    L.check(L.lib().hs_selftest_bounded_wait(ctypes.c_void_p(status.data_ptr()), 1 << 16,
                                             D.stream_handle()), "hs_selftest_bounded_wait")
    torch.cuda.synchronize()
    assert int(status.item()) == L.HS_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 60
    # the next launches run normally
    inputs = make_inputs(MIXED[:3])
    cfg = L.make_config(sweeps_per_pass=4)
    plan = run_plan(MIXED[:3], cfg, inputs)
    I0, I1 = inputs[2]
    u, v = D.hs_forward(D.as_plane(torch.from_numpy(I0).cuda()), D.as_plane(torch.from_numpy(I1).cuda()),
                        MIXED[2][2], MIXED[2][3], cfg)
    assert_bitexact(plan.u[2].cpu().numpy(), u.cpu().numpy())


def test_batched_large_pair_auto_layout_equals_per_pair(cuda):
    """A batch holding a pair above the size where the per-pass kernels switch to 4 columns
    per lane: the batch (2 columns per lane unless asked otherwise) equals each pair's
    forward, which runs in the 4-column layout."""
    specs = [(1100, 1900, 1.1, 14), (65, 127, 1.7, 40), (1, 1, 1.0, 3), (240, 320, 0.9, 21)]
    inputs = make_inputs(specs, 4000)
    cfg = L.make_config(sweeps_per_pass=4, fast_math=True)
    plan = run_plan(specs, cfg, inputs)
    auto = L.make_config(sweeps_per_pass=4, fast_math=True, layout=0)
    for i, ((H, W, alpha, iters), (I0, I1)) in enumerate(zip(specs, inputs)):
        u, v = D.hs_forward(D.as_plane(torch.from_numpy(I0).cuda()),
                            D.as_plane(torch.from_numpy(I1).cuda()), alpha, iters, auto)
        torch.cuda.synchronize()
        assert_bitexact(plan.u[i].cpu().numpy(), u.cpu().numpy(), f"u pair {i}")
        assert_bitexact(plan.v[i].cpu().numpy(), v.cpu().numpy(), f"v pair {i}")
