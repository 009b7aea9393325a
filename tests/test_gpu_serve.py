"""Serving loop: continuous batching, admission by resource profile and device memory budget."""
import threading
import time

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _cfg(preset="secure"):
    import stwo_b200 as sb
    c = oracle.config(preset)
    return sb.PcsConfig(c.pow_bits, sb.FriConfig(c.log_blowup_factor, c.log_last_layer_degree_bound, c.n_queries))


def _stream(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        out.append(dict(log_n=int(rng.integers(12, 21)), W=int(rng.choice([16, 32, 100])),
                        trace_seed=int(rng.integers(1, 2**62)), channel_seed=int(rng.integers(0, 2**62)),
                        gap_s=float(rng.exponential(1 / 200.0))))
    return out


def test_served_proofs_equal_their_single_runs(ctx):
    import stwo_b200 as sb
    g = _cfg()
    reqs = _stream(7, 24)
    tickets = [None] * len(reqs)
    with sb.Server(ctx, slots=6, profile=2) as srv:
        def producer():
            for i, r in enumerate(reqs):
                tickets[i] = srv.submit(sb.Statement(r["log_n"], r["W"]), g, trace_kind=sb.TRACE_SEEDED,
                                        trace_seed=r["trace_seed"], channel_seed=r["channel_seed"])
                time.sleep(r["gap_s"])
        th = threading.Thread(target=producer)
        th.start()
        served = []
        for i in range(len(reqs)):
            while tickets[i] is None:
                time.sleep(0.001)
            served.append(srv.wait(tickets[i]))
        th.join()
        snap = srv.snapshot()
    assert snap["completed"] == len(reqs) and snap["failed"] == 0
    assert snap["peak_in_flight"] > 1  # requests overlapped on the device
    for r, (proof, stats) in zip(reqs, served):
        alone = ctx.prove_wide_fibonacci(sb.Statement(r["log_n"], r["W"]), g, trace_kind=sb.TRACE_SEEDED,
                                         trace_seed=r["trace_seed"], channel_seed=r["channel_seed"])
        assert proof == alone
        assert stats["accounted_bytes"] == 16 * r["W"] << r["log_n"]


def test_served_proofs_equal_the_oracle(ctx):
    """Served proofs of mixed shapes and presets, in flight together, against the oracle's bytes."""
    import stwo_b200 as sb
    rng = np.random.default_rng(31)
    reqs = [dict(log_n=int(rng.integers(12, 17)), W=int(rng.choice([16, 32, 100])), preset=p,
                 trace_seed=int(rng.integers(1, 2**62)), channel_seed=int(rng.integers(0, 2**62)))
            for p in ("secure", "functional", "secure", "functional", "secure", "functional")]
    with sb.Server(ctx, slots=4, profile=2) as srv:
        tickets = [srv.submit(sb.Statement(r["log_n"], r["W"]), _cfg(r["preset"]), trace_kind=sb.TRACE_SEEDED,
                              trace_seed=r["trace_seed"], channel_seed=r["channel_seed"]) for r in reqs]
        served = [srv.wait(t)[0] for t in tickets]
        assert srv.snapshot()["peak_in_flight"] > 1
    for r, proof in zip(reqs, served):
        assert proof == oracle.prove_wide_fib(r["log_n"], r["W"], oracle.config(r["preset"]), trace_kind=1,
                                              trace_seed=r["trace_seed"], channel_seed=r["channel_seed"]), r


def test_resource_profile_admission(ctx):
    import stwo_b200 as sb
    g = _cfg("functional")
    cases = [(0, 18, 100, True), (0, 20, 100, False), (1, 20, 100, True), (1, 21, 100, False),
             (1, 22, 100, False), (2, 22, 100, True), (2, 22, 101, False)]
    for profile, log_n, W, ok in cases:
        with sb.Server(ctx, slots=1, profile=profile) as srv:
            if ok:
                t = srv.submit(sb.Statement(log_n, W), g, trace_kind=sb.TRACE_SEEDED, trace_seed=1)
                proof, _ = srv.wait(t)
                assert len(proof) > 0
            else:
                with pytest.raises(sb.StwoError) as e:
                    srv.submit(sb.Statement(log_n, W), g, trace_kind=sb.TRACE_SEEDED, trace_seed=1)
                assert e.value.status == sb.E_REJECTED


def test_memory_budget_limits_in_flight_work(ctx):
    import stwo_b200 as sb
    g = _cfg("functional")
    with sb.Server(ctx, slots=2, profile=1) as probe:
        _, st = probe.wait(probe.submit(sb.Statement(16, 32), g, trace_kind=sb.TRACE_SEEDED, trace_seed=1))
    ws = st["workspace_bytes"]
    with sb.Server(ctx, slots=4, profile=1, memory_budget=ws + ws // 2) as srv:
        ts = [srv.submit(sb.Statement(16, 32), g, trace_kind=sb.TRACE_SEEDED, trace_seed=10 + i) for i in range(5)]
        proofs = [srv.wait(t)[0] for t in ts]
        with pytest.raises(sb.StwoError) as e:
            srv.submit(sb.Statement(18, 32), g, trace_kind=sb.TRACE_SEEDED, trace_seed=1)
        assert e.value.status == sb.E_REJECTED
        snap = srv.snapshot()
    assert snap["peak_in_flight"] == 1 and snap["peak_workspace_bytes"] <= ws + ws // 2
    for i, p in enumerate(proofs):
        assert p == ctx.prove_wide_fibonacci(sb.Statement(16, 32), g, trace_kind=sb.TRACE_SEEDED, trace_seed=10 + i)


def test_close_finishes_queued_requests(ctx):
    import stwo_b200 as sb
    g = _cfg("functional")
    srv = sb.Server(ctx, slots=2, profile=1)
    for i in range(6):
        srv.submit(sb.Statement(14, 16), g, trace_kind=sb.TRACE_SEEDED, trace_seed=i)
    srv.close()  # drains without a wait per request


def test_served_mix_with_xor_lookups(ctx):
    """70% wide-Fibonacci and 30% LogUp XOR-lookup requests through one serving loop: every proof
    equals its single run, and the XOR proofs verify."""
    import stwo_b200 as sb
    import verifier
    g = _cfg()
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(16):
        if rng.random() < 0.3:
            reqs.append(("xor", int(rng.integers(12, 17)), int(rng.integers(1, 2**40))))
        else:
            reqs.append(("wf", int(rng.integers(12, 17)), int(rng.choice([16, 32, 100])), int(rng.integers(1, 2**40))))
    if not any(r[0] == "xor" for r in reqs):
        reqs[0] = ("xor", 14, 5)
    with sb.Server(ctx, slots=4, profile=2) as srv:
        tickets = []
        for r in reqs:
            if r[0] == "xor":
                tickets.append(srv.submit_xor(r[1], g, seed=r[2]))
            else:
                tickets.append(srv.submit(sb.Statement(r[1], r[2]), g, trace_kind=sb.TRACE_SEEDED, trace_seed=r[3]))
        served = [srv.wait(t)[0] for t in tickets]
    for r, p in zip(reqs, served):
        if r[0] == "xor":
            assert p == ctx.prove_logup_xor(r[1], g, seed=r[2])
            assert verifier.verify_logup_xor(p, r[1], 16)
        else:
            assert p == ctx.prove_wide_fibonacci(sb.Statement(r[1], r[2]), g, trace_kind=sb.TRACE_SEEDED,
                                                 trace_seed=r[3])


def test_served_first_column_traces(ctx):
    """Requests that hand the server only col0/col1 from host memory (TRACE_FIRST_COLUMNS): the
    buffers are read when a slot runs the request; proofs equal the seeded single runs."""
    import stwo_b200 as sb
    import torch
    g = _cfg("functional")
    shapes = [(14, 32, 3), (16, 100, 4), (12, 16, 5), (15, 17, 6)]
    twos = []
    for log_n, W, seed in shapes:
        full = torch.empty(W << log_n, dtype=torch.int32, device="cuda")
        ctx.wide_fib_trace(full, log_n, W, sb.TRACE_SEEDED, seed)
        twos.append(full[: 2 << log_n].cpu().numpy().view(np.uint32).reshape(2, -1).copy())
    with sb.Server(ctx, slots=3, profile=1) as srv:
        ts = [srv.submit(sb.Statement(n, W), g, trace=two, trace_kind=sb.TRACE_FIRST_COLUMNS)
              for (n, W, _), two in zip(shapes, twos)]
        out = [srv.wait(t)[0] for t in ts]
    for (n, W, seed), p in zip(shapes, out):
        assert p == ctx.prove_wide_fibonacci(sb.Statement(n, W), g, trace_kind=sb.TRACE_SEEDED, trace_seed=seed)


def test_warmup_presizes_slots(ctx):
    import stwo_b200 as sb
    g = _cfg("functional")
    with sb.Server(ctx, slots=3, profile=1, persistent_workspaces=True) as srv:
        srv.warmup(16, 32, 1, 12)
        held = srv.snapshot()["peak_workspace_bytes"]
        assert held > 0
        ts = [srv.submit(sb.Statement(16, 32), g, trace_kind=sb.TRACE_SEEDED, trace_seed=i) for i in range(3)]
        ts.append(srv.submit_xor(12, g, seed=1))
        out = [srv.wait(t)[0] for t in ts]
    assert out[0] == ctx.prove_wide_fibonacci(sb.Statement(16, 32), g, trace_kind=sb.TRACE_SEEDED, trace_seed=0)
    assert out[3] == ctx.prove_logup_xor(12, g, seed=1)


def test_server_verifies_every_proof(ctx):
    import stwo_b200 as sb
    g = _cfg("functional")
    with sb.Server(ctx, slots=3, profile=2, verify=True) as srv:
        ts = [srv.submit(sb.Statement(12 + i, 16), g, trace_kind=sb.TRACE_SEEDED, trace_seed=i) for i in range(4)]
        ts.append(srv.submit_xor(12, g, seed=9))
        outs = [srv.wait(t)[0] for t in ts]
    for i in range(4):
        assert sb.verify_wide_fibonacci(outs[i], 12 + i, 16)
    assert sb.verify_logup_xor(outs[4], 12)
