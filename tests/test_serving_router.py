"""Host routing of the multi-GPU request loop (CPU only): one engine per GPU
behind a router that sends each request to the device with the least
outstanding work.  The engines here are fakes that complete requests on the
host, so the routing, the load accounting and the mapping of results back to
their device are tested without a GPU."""
import threading
import types

import pytest

from vortexstark_b200.serving import MultiGpuServer


class FakeEngine:
    def __init__(self, device, fail_on=None, **kw):
        self.device, self.kw, self.fail_on = device, kw, fail_on
        self.lock = threading.Lock()
        self.pending, self.done, self.closed = [], {}, False

    def submit(self, tag, log_n, a, b):
        if self.fail_on is not None and tag == self.fail_on:
            raise RuntimeError("submit refused")
        with self.lock:
            self.pending.append((tag, log_n))

    def poll(self, max_items=256, wait_ms=0):
        with self.lock:
            take, self.pending = self.pending[:max_items], self.pending[max_items:]
            for tag, _ in take:
                self.done[tag] = f"{self.device}:{tag}".encode()
        return [types.SimpleNamespace(tag=t, log_n=ln, status=0) for t, ln in take]

    def result(self, tag, keep=True):
        with self.lock:
            v = self.done.pop(tag)
        return v if keep else None

    def close(self):
        self.closed = True


def _router(n=2, **kw):
    return MultiGpuServer(list(range(n)), budget_bytes=1 << 30, server_factory=lambda d, **k: FakeEngine(d, **kw))


def test_large_request_sends_small_ones_elsewhere():
    r = _router(2)
    assert r.submit(1, 24, 1, 2) == 0          # 2^26 points on device 0
    assert [r.submit(t, 16, 1, 2) for t in range(2, 10)] == [1] * 8  # 8 x 2^18 points stay below it
    assert r.outstanding() == [1 << 26, 8 << 18]
    got = r.poll()
    assert sorted(int(c.tag) for c in got) == list(range(1, 10))
    assert r.outstanding() == [0, 0]
    assert r.result(1) == b"0:1" and r.result(5) == b"1:5"


def test_balanced_when_sizes_are_equal():
    r = _router(4)
    devs = [r.submit(t, 20, 3, 4) for t in range(12)]
    assert devs == [0, 1, 2, 3] * 3
    assert r.device_of(7) == 3


def test_duplicate_tag_and_failed_submit_leave_no_load():
    r = MultiGpuServer([0, 1], budget_bytes=1, server_factory=lambda d, **k: FakeEngine(d, fail_on=5))
    r.submit(4, 18, 1, 1)
    with pytest.raises(ValueError):
        r.submit(4, 18, 1, 1)
    with pytest.raises(RuntimeError):
        r.submit(5, 18, 1, 1)
    assert sum(r.outstanding()) == 1 << 20
    r.poll()
    assert r.outstanding() == [0, 0]
    r.close()
    assert all(s.closed for s in r._servers)


def test_concurrent_submit_and_poll():
    r = _router(3)
    n = 600
    seen = []

    def submitter():
        for t in range(n):
            r.submit(t, 16 + 2 * (t % 5), t, t + 1)

    th = threading.Thread(target=submitter)
    th.start()
    while len(seen) < n:
        for c in r.poll(64, wait_ms=1):
            seen.append(int(c.tag))
            dev = r.device_of(int(c.tag))
            assert r.result(int(c.tag)) == f"{dev}:{int(c.tag)}".encode()
    th.join()
    assert sorted(seen) == list(range(n))
    assert r.outstanding() == [0, 0, 0]
