"""Serving form: a request loop over the device path with continuous batching.

Requests (compress a device-resident field, or decompress a device-resident stream) arrive as they
come; a request is admitted as soon as a worker slot is free and its device-memory estimate fits
the budget, and admitted requests run concurrently, each on a worker with its own library
context (a CUDA stream and scratch), so a request that arrives while others are on the GPU starts
on the GPU beside them.  Every request runs the same per-field path as a single
falcons_compress_device / falcons_decompress_device call, so its result is the same bits alone
and in the mix.

    srv = Server(workers=8, budget_bytes=120 << 30)
    fut = srv.submit_compress(x, config)        # -> Future of (stream tensor, stored config)
    fut = srv.submit_decompress(stream, dtype)   # -> Future of (flat field tensor, config)
    stats = open_loop(srv, requests, rate)       # Poisson arrivals; p50/p95/p99 latency, GB/s

The loop's own work is host-side bookkeeping; every byte of compression runs in the CUDA
kernels of libfalcons_b200.so (there is no CPU path)."""
from __future__ import annotations

import collections
import ctypes
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from . import device as D


def request_bytes(kind: str, nbytes: int) -> int:
    """Device memory a request holds while it runs: its input and output plus the path's scratch
    (codes, the unpredictable list, escape slots and entropy scratch, about 3x the field)."""
    return 4 * nbytes if kind == "compress" else 3 * nbytes


@dataclass(order=True)
class _Req:
    arrival: float
    seq: int
    kind: str = field(compare=False)
    nbytes: int = field(compare=False)
    args: tuple = field(compare=False)
    fut: Future = field(compare=False)
    ready: object = field(default=None, compare=False)  # CUDA event: the caller's work on the input is done
    start: float = field(default=0.0, compare=False)
    done: float = field(default=0.0, compare=False)


class Server:
    """Continuous-batching request loop: `workers` slots, each a host thread with its own library
    context and CUDA stream for the server's lifetime; a free slot takes the head of the FIFO queue
    as soon as its device-memory estimate fits the budget (a request waits while the head of the
    queue does not fit)."""

    def __init__(self, workers: int = 8, budget_bytes: int = 120 << 30, device: int = 0):
        self.device = device
        self.budget = int(budget_bytes)
        self.in_use = 0
        self._cv = threading.Condition()
        self._queue: collections.deque[_Req] = collections.deque()
        self._seq = 0
        self._stop = False
        self._ctxs = [_lib.Context(device) for _ in range(workers)]
        self.completed: list[_Req] = []
        self._threads = [threading.Thread(target=self._worker, args=(w,), daemon=True) for w in range(workers)]
        for t in self._threads:
            t.start()

    # ---- submission
    def submit_compress(self, x: torch.Tensor, config, arrival: float | None = None) -> Future:
        return self._submit("compress", x.numel() * x.element_size(), (x, config), arrival)

    def submit_decompress(self, stream: torch.Tensor, dtype, arrival: float | None = None,
                          num: int | None = None) -> Future:
        """`num`: the field's element count when the caller knows it (from the stream's header,
        `api.read_config`); otherwise it is read here, one small device-to-host copy."""
        if num is None:
            head = stream[:256].cpu().numpy().tobytes()
            c = _lib.Config()
            buf = bytearray(head)
            _lib.check(_lib.lib().falcons_read_config((ctypes.c_char * len(buf)).from_buffer(buf),
                                                      ctypes.c_size_t(len(buf)), ctypes.byref(c)), "read_config")
            num = int(c.num)
        nbytes = int(num) * torch.empty((), dtype=dtype).element_size()
        return self._submit("decompress", nbytes, (stream, dtype, int(num)), arrival)

    def _submit(self, kind, nbytes, args, arrival):
        fut = Future()
        need = request_bytes(kind, nbytes)
        if need > self.budget:
            fut.set_exception(ValueError(f"request needs {need} bytes, more than the {self.budget}-byte budget"))
            return fut
        # the input was written on the caller's stream; the worker's stream waits for it
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream(self.device))
        with self._cv:
            if self._stop:
                fut.set_exception(RuntimeError("server closed"))
                return fut
            self._seq += 1
            r = _Req(time.perf_counter() if arrival is None else arrival, self._seq, kind, nbytes, args, fut, ready)
            self._queue.append(r)
            self._cv.notify_all()
        return fut

    # ---- a worker slot: take the head of the queue when it fits the budget, run it, repeat
    def _admissible(self) -> bool:
        return bool(self._queue) and self.in_use + request_bytes(self._queue[0].kind, self._queue[0].nbytes) <= self.budget

    def _worker(self, w: int):
        ctx = self._ctxs[w]
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream(device=self.device)
        while True:
            with self._cv:
                while not self._admissible() and not (self._stop and not self._queue):
                    self._cv.wait()
                if not self._queue:
                    return
                r = self._queue.popleft()
                need = request_bytes(r.kind, r.nbytes)
                self.in_use += need
            r.start = time.perf_counter()
            try:
                stream.wait_event(r.ready)
                with torch.cuda.stream(stream):
                    if r.kind == "compress":
                        x, config = r.args
                        result = D.compress(x, config, ctx=ctx, stream=stream)
                    else:
                        s, dtype, num = r.args
                        out = torch.empty(num, dtype=dtype, device=s.device)
                        result = D.decompress(s, dtype, out=out, ctx=ctx, stream=stream)
                stream.synchronize()
                r.done = time.perf_counter()
                r.fut.set_result(result)
            except Exception as e:  # the request fails alone; the loop goes on
                r.done = time.perf_counter()
                r.fut.set_exception(e)
            with self._cv:
                self.in_use -= need
                self.completed.append(r)
                self._cv.notify_all()

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join(timeout=60)
        for c in self._ctxs:
            c.close()


def latency_stats(reqs) -> dict:
    lat = np.array([r.done - r.arrival for r in reqs]) * 1e3
    if lat.size == 0:
        return {}
    return {"n": int(lat.size), "p50_ms": float(np.percentile(lat, 50)), "p95_ms": float(np.percentile(lat, 95)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean())}


def open_loop(srv: Server, requests, rate: float, seed: int = 0):
    """Submits `requests` (callables that submit one request given its arrival time) with Poisson
    arrivals at `rate` per second, waits for all, and returns (futures, wall seconds)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=len(requests))
    t0 = time.perf_counter()
    due = t0
    futs = []
    for make, gap in zip(requests, gaps):
        due += gap
        now = time.perf_counter()
        if due > now:
            time.sleep(due - now)
        futs.append(make(due))
    for f in futs:
        try:
            f.result()
        except Exception:
            pass
    return futs, time.perf_counter() - t0
