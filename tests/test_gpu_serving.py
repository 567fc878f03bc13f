"""Serving engine: continuous batching must not change any proof byte.

Every request's proof, computed while other requests of other sizes are in
flight on the same GPU, must equal the proof of the same request computed
alone (and the oracle's).  A tight memory budget forces queueing and slot
reuse; that must not change any byte either.
"""
import pytest

from vortexstark_b200 import prover
from vortexstark_b200.serving import ProofServer, poisson_arrivals, run_stream
from vortexstark_b200.workload import SplitMix64

pytestmark = pytest.mark.gpu


def _stream(seed, n, sizes):
    g = SplitMix64(seed)
    return [(sizes[g.next() % len(sizes)], g.m31(), g.m31()) for _ in range(n)]


def test_mixed_stream_equals_alone(oracle):
    reqs = _stream(7, 40, [8, 10, 12, 14, 16])
    with ProofServer(budget_bytes=8 << 30, max_inflight=8) as srv:
        for s in (8, 10, 12, 14, 16):
            srv.prewarm(s, 2)
        summary, results = run_stream(srv, reqs, poisson_arrivals(len(reqs), 2000.0, 1), keep_results=True)
    assert summary["n"] == len(reqs)
    for i, (log_n, a, b) in enumerate(reqs):
        alone = prover.prove_bytes(a, b, log_n)
        assert results[i] == alone, (i, log_n)
        if log_n <= 12:
            assert alone == oracle.prove(a, b, log_n)


def test_measured_mix_equals_alone(oracle):
    """The benchmark's own stream (log_n 16..24 at weights .4/.25/.2/.1/.05),
    with three requests of each large size added, through the engine as the
    benchmark configures it and at an arrival rate above the plain path's
    capacity, so large and small proofs overlap on the device.  Every proof
    equals the same request proved alone; the log_n = 16 ones equal the
    oracle's."""
    from vortexstark_b200.workload import served_stream

    reqs = served_stream(2024, 40)
    g = SplitMix64(99)
    reqs += [(ln, g.m31(), g.m31()) for ln in (20, 22, 24) for _ in range(3)]
    g2 = SplitMix64(5)
    order = sorted(range(len(reqs)), key=lambda i: g2.next())
    reqs = [reqs[i] for i in order]
    with ProofServer(budget_bytes=48 << 30, max_inflight=24) as srv:
        for ln, c in {16: 6, 18: 4, 20: 3, 22: 2, 24: 2}.items():
            srv.prewarm(ln, c)
        summary, results = run_stream(srv, reqs, poisson_arrivals(len(reqs), 600.0, 3), keep_results=True)
    assert summary["n"] == len(reqs)
    assert {ln for ln, _, _ in reqs} >= {16, 18, 20, 22, 24}
    for i, (log_n, a, b) in enumerate(reqs):
        alone = prover.prove_bytes(a, b, log_n)
        assert results[i] == alone, (i, log_n)
        if log_n == 16:
            assert alone == oracle.prove(a, b, log_n)


def test_tight_budget_queues_and_stays_exact():
    reqs = _stream(11, 16, [10, 12])
    # room for one slot of each size (slot buffers + device input words +
    # the size's tables) and half a slot more: every other request queues
    slot, tab = {}, {}
    for ln in (10, 12):
        c = prover.ProverCache(ln)
        slot[ln], tab[ln] = c.slot_bytes() + 256, c.table_bytes()
        c.close()
    budget = sum(slot.values()) + sum(tab.values()) + min(slot.values()) // 2
    with ProofServer(budget_bytes=budget, max_inflight=4) as srv:
        summary, results = run_stream(srv, reqs, [0.0] * len(reqs), keep_results=True)
        st = srv.stats()
    assert st["bytes_used"] <= budget and st["slots"] == 2
    for i, (log_n, a, b) in enumerate(reqs):
        assert results[i] == prover.prove_bytes(a, b, log_n)


def test_burst_while_slots_are_created():
    # no prewarm: the engine creates slots (lock released) while the
    # submitter keeps appending requests
    reqs = _stream(17, 96, [8, 9, 10, 11])
    with ProofServer(budget_bytes=4 << 30, max_inflight=16) as srv:
        summary, results = run_stream(srv, reqs, [0.0] * len(reqs), keep_results=True)
        st = srv.stats()
    assert summary["n"] == len(reqs) and st["pending"] == 0 and st["inflight"] == 0
    for i, (log_n, a, b) in enumerate(reqs):
        assert results[i] == prover.prove_bytes(a, b, log_n), (i, log_n)


def test_plain_launches_without_graphs():
    reqs = _stream(13, 8, [10, 11])
    with ProofServer(budget_bytes=1 << 30, max_inflight=4, use_graphs=False) as srv:
        summary, results = run_stream(srv, reqs, [0.0] * len(reqs), keep_results=True)
    for i, (log_n, a, b) in enumerate(reqs):
        assert results[i] == prover.prove_bytes(a, b, log_n)


def test_multi_engine_router_equals_alone(oracle):
    """The multi-GPU request loop's router over two engines (here both on
    GPU 0; a node gives each its own GPU): every proof equals the same
    request proved alone, whichever engine ran it."""
    from vortexstark_b200.serving import MultiGpuServer

    reqs = _stream(23, 24, [10, 12, 14, 16])
    with MultiGpuServer([0, 0], budget_bytes=4 << 30, max_inflight=8) as srv:
        summary, results = run_stream(srv, reqs, poisson_arrivals(len(reqs), 3000.0, 2), keep_results=True)
    assert summary["n"] == len(reqs)
    for i, (log_n, a, b) in enumerate(reqs):
        assert results[i] == prover.prove_bytes(a, b, log_n), (i, log_n)
    assert results[0] == oracle.prove(reqs[0][1], reqs[0][2], reqs[0][0])


@pytest.mark.parametrize("split", [True, False])
def test_policy_knobs_validated_and_bytes_unchanged(split):
    """vx_server_set_policy rejects bad values and calls after the first
    slot exists; a non-default policy changes scheduling only, with large
    proofs (here log_n 12, 2^14 points) as head + tail graphs or whole."""
    from vortexstark_b200 import _lib

    with ProofServer(budget_bytes=1 << 30, max_inflight=4) as srv:
        for kw in (dict(priority=4), dict(max_large=0), dict(large_log_eval=0), dict(large_log_eval=40)):
            with pytest.raises(_lib.VortexError):
                srv.set_policy(**kw)
        srv.set_policy(large_log_eval=14, max_large=1, priority=3, small_cap=2, large_per_size=True,
                       split_large=split)
        srv.prewarm(10, 1)
        with pytest.raises(_lib.VortexError):
            srv.set_policy()
        reqs = _stream(29, 12, [8, 10, 12])
        summary, results = run_stream(srv, reqs, [0.0] * len(reqs), keep_results=True)
    for i, (log_n, a, b) in enumerate(reqs):
        assert results[i] == prover.prove_bytes(a, b, log_n), (i, log_n)


@pytest.mark.parametrize("smallest_first", [False, True])
def test_large_queue_order(smallest_first):
    """Waiting large proofs take the free large place oldest first, or
    smallest first (vx_server_set_queue_order): a 2^24-point proof runs
    while three smaller large proofs queue behind it; their start order
    follows the rule, and every proof equals the same request proved alone."""
    import time

    reqs = [(22, 11, 12), (14, 13, 14), (12, 15, 16), (13, 17, 18)]
    with ProofServer(budget_bytes=8 << 30, max_inflight=8) as srv:
        srv.set_policy(large_log_eval=14)  # log_n >= 12 is large
        srv.set_queue_order(smallest_first=smallest_first)
        for s in (22, 14, 12, 13):
            srv.prewarm(s, 1)
        srv.submit(0, *reqs[0])
        t0 = time.time()
        while srv.stats()["inflight"] == 0 and time.time() - t0 < 5:
            time.sleep(0.0001)
        for i in (1, 2, 3):  # queued while the 2^24-point proof's head runs (about 4 ms)
            srv.submit(i, *reqs[i])
        done = {}
        while len(done) < 4:
            for c in srv.poll(8, wait_ms=100):
                assert c.status == 0
                done[int(c.tag)] = (c.start_ns, srv.result(int(c.tag)))
    order = [t for t, _ in sorted(done.items(), key=lambda kv: kv[1][0])]
    assert order == ([0, 2, 3, 1] if smallest_first else [0, 1, 2, 3])
    for i, (log_n, a, b) in enumerate(reqs):
        assert done[i][1] == prover.prove_bytes(a, b, log_n), i
