"""Serving: continuous batching of mixed-size Fibonacci proof requests.

``ProofServer`` wraps the native serving engine (vx_server_* in
libvortex_b200): requests queue on the host, a dispatcher thread admits them
as proof slots of their size free up or fit in the device-memory budget, and
up to ``max_inflight`` proofs overlap on the GPU, each as one CUDA graph on
its own stream.  ``run_stream`` replays a request stream with Poisson
arrivals and reports throughput and latency; ``run_sequential`` is the plain
one-proof-at-a-time path on the same arrivals, for comparison.
"""
from __future__ import annotations

import ctypes as C
import random
import statistics
import threading
import time

from . import _lib


class Completion(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("status", C.c_int32), ("log_n", C.c_uint32), ("submit_ns", C.c_uint64),
                ("start_ns", C.c_uint64), ("done_ns", C.c_uint64), ("proof_bytes", C.c_uint64)]


class ProofServer:
    def __init__(self, budget_bytes: int, max_inflight: int = 16, blowup_bits: int = 2, n_queries: int = 80,
                 use_graphs: bool = True):
        self._s = C.c_void_p()
        self._blowup_bits, self._n_queries = blowup_bits, n_queries
        self._log_n = {}
        _lib.check(_lib.lib().vx_server_create(int(budget_bytes), max_inflight, blowup_bits, n_queries,
                                               1 if use_graphs else 0, C.byref(self._s)))

    def set_policy(self, large_log_eval: int = 24, max_large: int = 1, priority: int = 0,
                   small_cap: int = 0, large_per_size: bool = False, split_large: bool = True) -> None:
        """Scheduling policy (before the first prewarm or submit): proofs of at
        least 2^large_log_eval evaluation points are large, at most max_large
        of them in flight (per size if large_per_size); priority 0 = small
        proofs first, 1 = equal, 2 = large proofs first, 3 = graded by size;
        small_cap bounds small proofs in flight beside a large one (0 = none);
        split_large runs a large proof's latency-bound tail on a high-priority
        stream outside the max_large count, overlapping the next one's head."""
        _lib.check(_lib.lib().vx_server_set_policy(self._s, large_log_eval, max_large, priority, small_cap,
                                                   1 if large_per_size else 0, 1 if split_large else 0))

    def set_queue_order(self, smallest_first: bool = False, max_wait_ms: float = 0.0) -> None:
        """Order of waiting large proofs: oldest first, or the smallest first
        with the oldest going first once it has waited max_wait_ms (0 = never)."""
        _lib.check(_lib.lib().vx_server_set_queue_order(self._s, 1 if smallest_first else 0,
                                                        int(round(max_wait_ms * 1000))))

    def prewarm(self, log_n: int, count: int) -> None:
        _lib.check(_lib.lib().vx_server_prewarm(self._s, log_n, count))

    def submit(self, tag: int, log_n: int, a: int, b: int) -> None:
        self._log_n[tag] = log_n  # before the engine can complete it
        try:
            _lib.check(_lib.lib().vx_server_submit(self._s, tag, log_n, a, b))
        except Exception:
            self._log_n.pop(tag, None)
            raise

    def poll(self, max_items: int = 256, wait_ms: int = 0):
        buf = (Completion * max_items)()
        n = C.c_uint32()
        _lib.check(_lib.lib().vx_server_poll(self._s, buf, max_items, C.byref(n), wait_ms))
        return [buf[i] for i in range(n.value)]

    def result(self, tag: int, keep: bool = True):
        """Proof bytes of a finished request (and release them)."""
        L = _lib.lib()
        n = C.c_size_t()
        log_n = self._log_n.pop(tag, None)
        if not keep:
            _lib.check(L.vx_server_result(self._s, tag, None, 0, C.byref(n)))
            return None
        if log_n is None:
            raise _lib.VortexError(f"vx_server_result: unknown tag {tag}")
        cap = int(L.vx_proof_size(log_n, self._blowup_bits, self._n_queries))
        buf = bytearray(cap)
        _lib.check(L.vx_server_result(self._s, tag, C.addressof((C.c_uint8 * cap).from_buffer(buf)), cap,
                                      C.byref(n)))
        return bytes(memoryview(buf)[: n.value])

    def stats(self) -> dict:
        ns, inf, pend = C.c_uint32(), C.c_uint32(), C.c_uint32()
        used = C.c_size_t()
        _lib.check(_lib.lib().vx_server_stats(self._s, C.byref(ns), C.byref(inf), C.byref(pend), C.byref(used)))
        return {"slots": ns.value, "inflight": inf.value, "pending": pend.value, "bytes_used": used.value}

    def close(self) -> None:
        if self._s:
            _lib.lib().vx_server_destroy(self._s)
            self._s = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_arrivals(n: int, rate: float, seed: int):
    """Arrival offsets (seconds) of a Poisson process with the given rate."""
    rng = random.Random(seed)
    t, out = 0.0, []
    for _ in range(n):
        t += rng.expovariate(rate)
        out.append(t)
    return out


def _pct(sorted_vals, q):
    return sorted_vals[min(len(sorted_vals) - 1, int(round(q * (len(sorted_vals) - 1))))]


def _summary(lat_ms, makespan_s, n, sizes=None):
    lat = sorted(lat_ms)
    out = {"proofs_per_s": n / makespan_s, "p50_ms": statistics.median(lat), "p99_ms": _pct(lat, 0.99),
           "mean_ms": statistics.fmean(lat), "makespan_s": makespan_s, "n": n, "lat_ms": list(lat_ms)}
    if sizes is not None:
        by = {}
        for ln in sorted(set(sizes)):
            v = sorted(x for x, s in zip(lat_ms, sizes) if s == ln)
            by[str(ln)] = {"n": len(v), "p50_ms": statistics.median(v), "p99_ms": _pct(v, 0.99)}
        out["by_log_n"] = by
    return out


def run_stream(server: ProofServer, requests, arrivals, keep_results: bool = False):
    """Submit requests (log_n, a, b) at the given arrival offsets; return the
    summary and, if asked, the proof bytes per request index."""
    n = len(requests)
    lat = [0.0] * n
    results = {}
    done = threading.Event()
    t0 = time.perf_counter_ns()
    submit_ns = [0] * n

    def submitter():
        for i, ((log_n, a, b), at) in enumerate(zip(requests, arrivals)):
            target = t0 + int(at * 1e9)
            while True:
                d = target - time.perf_counter_ns()
                if d <= 0:
                    break
                time.sleep(min(d / 1e9, 0.001) if d > 200_000 else 0)
            submit_ns[i] = time.perf_counter_ns()
            server.submit(i, log_n, a, b)

    th = threading.Thread(target=submitter)
    th.start()
    got = 0
    last_done = t0
    while got < n:
        for c in server.poll(256, wait_ms=50):
            if c.status != 0:
                raise RuntimeError(f"request {c.tag} failed with status {c.status}: {_lib.last_error()}")
            i = int(c.tag)
            lat[i] = (c.done_ns - c.submit_ns) / 1e6
            last_done = max(last_done, time.perf_counter_ns())
            if keep_results:
                results[i] = server.result(i)
            else:
                server.result(i, keep=False)
            got += 1
    th.join()
    done.set()
    s = _summary(lat, (last_done - t0) / 1e9, n, [r[0] for r in requests])
    return s, results


def plain_caches(sizes, blowup_bits: int = 2, n_queries: int = 80):
    """One device-resident ProverCache (slot + pinned host buffer) per size:
    the fastest one-proof-at-a-time path."""
    from . import prover

    return {ln: prover.ProverCache(ln, blowup_bits, n_queries) for ln in sorted(set(sizes))}


def run_sequential(requests, arrivals, blowup_bits: int = 2, n_queries: int = 80, caches=None):
    """The plain one-proof-at-a-time GPU path on the same arrivals: requests in
    arrival order, each started when it has arrived and the previous proof has
    finished, through one cached slot with a pinned host buffer per size
    (``prove_cached_bytes``)."""
    from . import prover

    n = len(requests)
    if caches is None:
        caches = plain_caches([r[0] for r in requests], blowup_bits, n_queries)
    lat = []
    t0 = time.perf_counter()
    for (log_n, a, b), at in zip(requests, arrivals):
        now = time.perf_counter() - t0
        if now < at:
            time.sleep(at - now)
        start_wait = t0 + at
        prover.prove_cached_bytes(a, b, caches[log_n])
        lat.append((time.perf_counter() - start_wait) * 1e3)
    return _summary(lat, time.perf_counter() - t0, n, [r[0] for r in requests])


class MultiGpuServer:
    """One serving engine per GPU behind a host router: the request loop of a
    node with several GPUs (no traffic between GPUs; every proof runs on one
    device).  A request goes to the device with the least outstanding work,
    counted as the evaluation points (2^(log_n + blowup_bits)) of its
    admitted, unfinished requests, so a GPU busy with a large proof takes the
    next small ones elsewhere.  Tags are global; completions and proof bytes
    come back from whichever device ran the request.

    ``server_factory(device, **kw)`` builds one engine; the default builds a
    ProofServer with that device current (its dispatcher thread keeps it)."""

    def __init__(self, devices, budget_bytes: int, max_inflight: int = 24, blowup_bits: int = 2,
                 n_queries: int = 80, use_graphs: bool = True, server_factory=None):
        if not devices:
            raise ValueError("MultiGpuServer needs at least one device")
        self._blowup_bits = blowup_bits
        factory = server_factory or _device_server
        self._servers = [factory(d, budget_bytes=budget_bytes, max_inflight=max_inflight, blowup_bits=blowup_bits,
                                 n_queries=n_queries, use_graphs=use_graphs) for d in devices]
        self._devices = list(devices)
        self._load = [0] * len(self._servers)
        self._where = {}    # tag -> server index, until its result is taken
        self._weight = {}   # tag -> points counted in _load, until it completes
        self._lock = threading.Lock()

    def pick(self, log_n: int) -> int:
        """Index of the device that takes the next request (least outstanding points; lowest index on ties)."""
        with self._lock:
            return min(range(len(self._load)), key=lambda i: (self._load[i], i))

    def submit(self, tag: int, log_n: int, a: int, b: int) -> int:
        w = 1 << (log_n + self._blowup_bits)
        with self._lock:
            if tag in self._where:
                raise ValueError(f"tag {tag} is already in use")
            i = min(range(len(self._load)), key=lambda k: (self._load[k], k))
            self._load[i] += w
            self._where[tag], self._weight[tag] = i, w
        try:
            self._servers[i].submit(tag, log_n, a, b)
        except Exception:
            with self._lock:
                self._load[i] -= w
                self._where.pop(tag, None)
                self._weight.pop(tag, None)
            raise
        return i

    def poll(self, max_items: int = 256, wait_ms: int = 0):
        """Completions from every device; waits up to wait_ms (split across
        the devices) only when none is ready."""
        out = []
        for s in self._servers:
            if len(out) < max_items:
                out += s.poll(max_items - len(out), 0)
        if not out and wait_ms > 0:
            per = max(1, wait_ms // len(self._servers))
            for s in self._servers:
                out += s.poll(max_items - len(out), per)
                if out:
                    break
        with self._lock:
            for c in out:
                tag = int(c.tag)
                i = self._where.get(tag)
                if i is not None:
                    self._load[i] -= self._weight.pop(tag, 0)
        return out

    def result(self, tag: int, keep: bool = True):
        with self._lock:
            i = self._where.pop(tag)
        return self._servers[i].result(tag, keep)

    def device_of(self, tag: int) -> int:
        with self._lock:
            return self._devices[self._where[tag]]

    def outstanding(self) -> list:
        with self._lock:
            return list(self._load)

    def close(self) -> None:
        for s in self._servers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _device_server(device: int, **kw) -> ProofServer:
    import torch

    with torch.cuda.device(device):
        return ProofServer(**kw)
