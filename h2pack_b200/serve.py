"""Served form: resident H2 matrices, continuous batching of matvec and PCG requests.

A :class:`Server` keeps several H2 images resident in HBM (admitted while their
device footprint fits a budget) and serves requests for (K + mu I) x = b solves and
(K + mu I) b products.  Each resident matrix has a device CG engine
(``h2gpu_cg_*``, include/h2gpu.h) with 16 slots: requests that arrive while others
run are admitted into free slots between batches of iterations, every iteration
applies the matrix once to the panel of all its slots (one H2 matmul), a finished
request frees its slot at once, and the engines of different matrices run on their
images' own streams, so their work overlaps on the device.

Engines are decoupled: the scheduler never waits on one engine while others could
run.  It polls every in-flight engine's completion (``h2gpu_cg_query``, an event
recorded after its enqueued iterations), collects an engine as soon as it is done and
relaunches it at once, so requests on a small matrix cycle at that matrix's pace and
never wait for the iterations of a large one.  A request may carry a deadline
(``timeout`` seconds after its arrival); past it, it is dropped from the queue or its
slot is cancelled (``h2gpu_cg_cancel``) and it is returned with status "timeout".

The solver is H2Pack's left-preconditioned CG (examples/PCG/pcg.c:11-152, identity
preconditioner, shift wrapper of examples/SPDHSS-H2/pcg_tests.c:13-20) in lock step
for the slots of an engine: FP64 vectors and inner products on the device, the
operator in the image's precision, and every ``refresh`` iterations (and whenever
the recursive residual claims convergence) the true residual b - (K + mu I) x
recomputed with the FP64 operator and CG restarted from it -- iterative refinement,
so a mixed-precision operator still reaches the FP64 tolerance.  The host enqueues
``iters_per_sync`` iterations per engine and reads the 16 slot records once after
them; it never waits per iteration.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import heapq
import time

import numpy as np
import torch

from . import _abi
from .h2pack import Image


@dataclasses.dataclass
class Request:
    rid: int
    matrix: str
    kind: str                  # "matvec" or "pcg"
    b: torch.Tensor            # device float64 vector of length N
    arrival: float = 0.0       # seconds from the start of the run
    tol: float = 1e-6
    max_iter: int = 5000
    timeout: float | None = None   # seconds after arrival; None: no deadline
    # filled by the server
    status: str = ""           # "done" or "timeout"
    x: torch.Tensor | None = None
    start: float | None = None
    finish: float | None = None
    iters: int = 0
    relres: float | None = None
    converged: bool = False
    history: list | None = None   # ||r||_2 after every CG iteration (Server.run(history=True))


class SlotBlock:
    """Up to 16 requests of one matrix advanced in lock step by its device CG engine."""

    def __init__(self, image: Image, mu: float, precision: str, max_slots: int, refresh: int,
                 iters_per_sync: int):
        self.img, self.lib, self.N = image, image.lib, image.N
        image.set_precision(precision)
        h = C.c_void_p()
        _abi.check(self.lib.h2gpu_cg_create(image.handle, float(mu), int(refresh), C.byref(h)), self.lib,
                   "h2gpu_cg_create")
        self.h = h
        self.S = max(1, min(int(max_slots), 16))
        self.k = max(1, int(iters_per_sync))
        self.req: list[Request | None] = [None] * 16
        self.free = list(range(self.S - 1, -1, -1))
        self.history = False
        self.need_check = False
        self.inflight = False
        self._st = (C.c_int * 16)()
        self._it = (C.c_int * 16)()
        self._rr = (C.c_double * 16)()

    def close(self):
        if self.h:
            self.lib.h2gpu_cg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass

    def busy(self) -> bool:
        return len(self.free) < self.S

    def admit(self, r: Request, now: float) -> bool:
        if not self.free:
            return False
        k = self.free.pop()
        self.req[k] = r
        r.start = now
        kind = _abi.CG_PCG if r.kind == "pcg" else _abi.CG_MATVEC
        _abi.check(self.lib.h2gpu_cg_admit(self.h, k, kind, C.c_void_p(r.b.data_ptr()), float(r.tol),
                                           int(r.max_iter)), self.lib, "h2gpu_cg_admit")
        return True

    def launch(self):
        """Enqueue (without waiting) the pending true-residual checks and k iterations."""
        if self.need_check:
            _abi.check(self.lib.h2gpu_cg_check(self.h), self.lib, "h2gpu_cg_check")
        _abi.check(self.lib.h2gpu_cg_step(self.h, self.k), self.lib, "h2gpu_cg_step")
        self.inflight = True

    def ready(self) -> bool:
        """True when the enqueued work has finished on the device (does not wait)."""
        st = self.lib.h2gpu_cg_query(self.h)
        if st < 0:
            _abi.check(st, self.lib, "h2gpu_cg_query")
        return st == 1

    def cancel(self, r: Request) -> bool:
        """Give up a request holding a slot; its slot is free for the next admission."""
        for k in range(16):
            if self.req[k] is r:
                _abi.check(self.lib.h2gpu_cg_cancel(self.h, k), self.lib, "h2gpu_cg_cancel")
                self.req[k] = None
                self.free.append(k)
                return True
        return False

    def requests(self) -> list:
        return [r for r in self.req if r is not None]

    def collect(self, now_fn, out: list):
        """Read the slot records of a finished engine, hand out finished requests, note
        slots awaiting a check."""
        _abi.check(self.lib.h2gpu_cg_sync(self.h, self._st, self._it, self._rr), self.lib, "h2gpu_cg_sync")
        self.inflight = False
        t = now_fn()
        self.need_check = False
        for k in range(16):
            r = self.req[k]
            if r is None:
                continue
            st = self._st[k]
            if st == _abi.CG_CHECK:
                self.need_check = True
            elif st == _abi.CG_DONE:
                x = torch.empty(self.N, dtype=torch.float64, device="cuda")
                _abi.check(self.lib.h2gpu_cg_take(self.h, k, C.c_void_p(x.data_ptr())), self.lib, "h2gpu_cg_take")
                r.x = x
                r.iters = int(self._it[k])
                if r.kind == "pcg":
                    r.relres = float(self._rr[k])
                    r.converged = r.relres <= r.tol
                    if self.history:
                        buf = np.zeros(max(1, r.iters))
                        n = self.lib.h2gpu_cg_history(self.h, k, buf.ctypes.data_as(C.POINTER(C.c_double)), len(buf))
                        r.history = [float(v) for v in buf[:max(0, n)]]
                r.finish = t
                r.status = "done"
                out.append(r)
                self.req[k] = None
                self.free.append(k)


class Server:
    """Resident matrices + continuous batching of matvec / PCG requests."""

    def __init__(self, budget_bytes: float = 150e9, max_slots: int = 16, refresh: int = 200,
                 iters_per_sync: int = 8):
        self.budget, self.max_slots, self.refresh = float(budget_bytes), min(int(max_slots), 16), refresh
        self.iters_per_sync = iters_per_sync
        self.blocks: dict[str, SlotBlock] = {}
        self.footprint: dict[str, float] = {}

    def used_bytes(self) -> float:
        return sum(self.footprint.values())

    def admit_matrix(self, name: str, image: Image, mu: float, precision: str = "mixed") -> bool:
        """Keep the image resident if its footprint (image + slot block) fits the budget."""
        st = image.stats()
        engine_bytes = 8.0 * image.N * 16 * 5          # b, x, r, p, Ap panels of the CG engine
        need = float(st["device_bytes"]) + engine_bytes
        if self.used_bytes() + need > self.budget:
            return False
        self.blocks[name] = SlotBlock(image, mu, precision, self.max_slots,
                                      self.refresh if precision != "fp64" else 0, self.iters_per_sync)
        self.footprint[name] = need
        return True

    def evict(self, name: str):
        blk = self.blocks.pop(name, None)
        if blk is not None:
            blk.close()
        self.footprint.pop(name, None)

    def run(self, requests: list[Request], realtime: bool = True, history: bool = False,
            poll_sleep: float = 50e-6) -> list[Request]:
        """Serve requests whose ``arrival`` offsets follow the wall clock (realtime) or
        are all present at time 0 (realtime=False).  Returns them in completion order.
        ``history`` records every PCG request's residual norm after each iteration.

        Each pass: arrivals join their matrix's FIFO queue; requests past their deadline
        leave (queue or slot); every in-flight engine whose work has finished is
        collected; queued requests take the free slots; every idle engine with busy
        slots is launched.  Nothing waits on one engine while another could make
        progress."""
        for blk in self.blocks.values():
            blk.history = history
        pending = [(r.arrival if realtime else 0.0, r.rid, r) for r in requests]
        heapq.heapify(pending)
        waiting: dict[str, list[Request]] = {n: [] for n in self.blocks}
        done: list[Request] = []
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        def expired(r, t):
            return r.timeout is not None and t - (r.arrival if realtime else 0.0) > r.timeout

        def give_up(r, t):
            r.finish, r.status = t, "timeout"
            done.append(r)

        # the right-hand sides were written on torch's stream; the engines read them on
        # their images' streams
        torch.cuda.current_stream().synchronize()
        while pending or any(waiting.values()) or any(b.busy() for b in self.blocks.values()):
            t = now()
            while pending and pending[0][0] <= t:
                _, _, r = heapq.heappop(pending)
                if r.matrix not in self.blocks:
                    raise KeyError(f"matrix {r.matrix!r} is not resident")
                waiting[r.matrix].append(r)
            for name, blk in self.blocks.items():
                q = waiting[name]
                for r in [r for r in q if expired(r, t)]:
                    q.remove(r)
                    give_up(r, t)
                for r in [r for r in blk.requests() if expired(r, t)]:
                    blk.cancel(r)
                    give_up(r, t)
            progressed = False
            for blk in self.blocks.values():      # collect every engine that has finished
                if blk.inflight and blk.ready():
                    blk.collect(now, done)
                    progressed = True
            t = now()
            for name, blk in self.blocks.items():  # freed slots take queued requests
                q = waiting[name]
                while q and blk.admit(q[0], t):
                    q.pop(0)
            for blk in self.blocks.values():      # relaunch idle engines at once
                if not blk.inflight and blk.busy():
                    blk.launch()
                    progressed = True
            if not progressed:
                nxt = pending[0][0] - now() if pending and not any(b.inflight for b in self.blocks.values()) else 0.0
                time.sleep(min(max(nxt, poll_sleep), 0.001))
        for blk in self.blocks.values():          # no engine keeps work in flight
            if blk.inflight:
                while not blk.ready():
                    time.sleep(poll_sleep)
                blk.collect(now, done)
        return done


def latency_stats(reqs: list[Request]) -> dict:
    """Latency percentiles and throughput of the requests served to completion (requests
    that timed out are counted separately)."""
    ok = [r for r in reqs if r.status != "timeout"]
    lat = np.array([r.finish - r.arrival for r in ok])
    span = max(r.finish for r in ok) - min(r.arrival for r in ok)
    return {"n": len(ok), "n_timeout": len(reqs) - len(ok), "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
            "throughput_req_s": len(ok) / span if span > 0 else None}
