"""Served form: resident H2 matrices, continuous batching of matvec and PCG requests.

A :class:`Server` keeps several H2 images resident in HBM (admitted while their
device footprint fits a budget) and serves requests for (K + mu I) x = b solves and
(K + mu I) b products.  Requests that arrive while others run are admitted into free
slots of their matrix's slot block at the next iteration boundary; every step applies
each busy matrix once to the panel of all its active slots (one device matmul of up
to ``max_slots`` right-hand sides), so the work of different requests overlaps on the
device.  A finished request frees its slot at once.

The solver is H2Pack's left-preconditioned CG (examples/PCG/pcg.c:11-152, identity
preconditioner, shift wrapper of examples/SPDHSS-H2/pcg_tests.c:13-20) run in lock
step for all slots of a block: FP64 vectors and inner products on the device, the
operator in the image's precision, and every ``refresh`` iterations (and before
declaring convergence) the true residual b - (K + mu I) x recomputed with the FP64
operator and CG restarted from it -- iterative refinement, so a mixed-precision
operator still reaches the FP64 tolerance (with an FP64 operator the true residual is
only recomputed when the recursive one claims convergence, as pcg.c:129-138 does once).
"""
from __future__ import annotations

import dataclasses
import heapq
import time

import numpy as np
import torch

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
    # filled by the server
    x: torch.Tensor | None = None
    start: float | None = None
    finish: float | None = None
    iters: int = 0
    relres: float | None = None
    converged: bool = False


class ShiftedOperator:
    """y = (K + mu I) x for device panels, K applied by an image in its precision and,
    for residual recomputation, in FP64 (the same image switched for that call)."""

    def __init__(self, image: Image, mu: float, precision: str):
        self.img, self.mu, self.precision = image, float(mu), precision
        self.N = image.N

    def apply(self, X: torch.Tensor, fp64: bool = False) -> torch.Tensor:
        if fp64 and self.precision != "fp64":
            self.img.set_precision("fp64")
            try:
                Y = self.img.matmul_device(X)
            finally:
                self.img.set_precision(self.precision)
        else:
            Y = self.img.matmul_device(X)
        return Y.add_(X, alpha=self.mu)


class SlotBlock:
    """Up to ``max_slots`` requests of one matrix advanced in lock step."""

    def __init__(self, op: ShiftedOperator, max_slots: int, refresh: int):
        self.op, self.S, self.refresh = op, max_slots, refresh
        N = op.N
        z = lambda: torch.zeros(N, max_slots, dtype=torch.float64, device="cuda")  # noqa: E731
        self.B, self.X, self.R, self.P = z(), z(), z(), z()
        self.rho = torch.ones(max_slots, dtype=torch.float64, device="cuda")
        self.bnorm = torch.ones(max_slots, dtype=torch.float64, device="cuda")
        self.req: list[Request | None] = [None] * max_slots
        self.it = [0] * max_slots          # iterations since the last restart
        self.free = list(range(max_slots))

    def busy(self) -> bool:
        return len(self.free) < self.S

    def admit(self, r: Request, now: float) -> bool:
        if not self.free:
            return False
        k = self.free.pop()
        self.req[k] = r
        r.start = now
        self.B[:, k] = r.b
        self.X[:, k] = 0.0
        self.R[:, k] = r.b                 # r = b - A*0
        self.P[:, k] = 0.0
        self.rho[k] = 1.0
        self.bnorm[k] = torch.linalg.vector_norm(r.b)
        self.it[k] = 0
        return True

    def _release(self, k: int, now: float, out: list):
        r = self.req[k]
        r.finish = now
        out.append(r)
        self.req[k] = None
        self.free.append(k)

    def step(self, now_fn, out: list):
        """One operator application for every active slot of the block."""
        act = [k for k in range(self.S) if self.req[k] is not None]
        if not act:
            return
        idx = torch.tensor(act, device="cuda")
        mv = [k for k in act if self.req[k].kind == "matvec"]
        cg = [k for k in act if self.req[k].kind == "pcg"]
        # panel: b for matvec slots, the CG direction for PCG slots
        if cg:
            cgi = torch.tensor(cg, device="cuda")
            # z = r (identity preconditioner); rho0 = rho; rho = r'z; p = z + beta p
            rho_new = (self.R[:, cgi] * self.R[:, cgi]).sum(0)
            first = torch.tensor([self.it[k] == 0 for k in cg], device="cuda")
            beta = torch.where(first, torch.zeros_like(rho_new), rho_new / self.rho[cgi])
            self.P[:, cgi] = self.R[:, cgi] + beta * self.P[:, cgi]
            self.rho[cgi] = rho_new
        panel = torch.empty(self.op.N, len(act), dtype=torch.float64, device="cuda")
        for j, k in enumerate(act):
            panel[:, j] = self.B[:, k] if self.req[k].kind == "matvec" else self.P[:, k]
        AP = self.op.apply(panel)
        col = {k: j for j, k in enumerate(act)}
        t = now_fn()
        for k in mv:
            r = self.req[k]
            r.x = AP[:, col[k]].clone()
            r.iters = 1
            self._release(k, t, out)
        if cg:
            cgi = torch.tensor(cg, device="cuda")
            S = AP[:, [col[k] for k in cg]]
            pAp = (self.P[:, cgi] * S).sum(0)
            alpha = self.rho[cgi] / pAp
            self.X[:, cgi] += alpha * self.P[:, cgi]
            self.R[:, cgi] -= alpha * S
            rn = torch.linalg.vector_norm(self.R[:, cgi], dim=0) / self.bnorm[cgi]
            rn_h = rn.cpu().numpy()
            refresh = []
            for j, k in enumerate(cg):
                self.it[k] += 1
                self.req[k].iters += 1
                periodic = self.op.precision != "fp64" and self.refresh > 0 and self.it[k] >= self.refresh
                if rn_h[j] <= self.req[k].tol or periodic or self.req[k].iters >= self.req[k].max_iter:
                    refresh.append(k)
            if refresh:
                self._refresh(refresh, now_fn, out)

    def _refresh(self, ks, now_fn, out):
        """True residual with the FP64 operator; converged slots leave, others restart CG."""
        ki = torch.tensor(ks, device="cuda")
        AX = self.op.apply(self.X[:, ki].contiguous(), fp64=True)
        Rt = self.B[:, ki] - AX
        rn = (torch.linalg.vector_norm(Rt, dim=0) / self.bnorm[ki]).cpu().numpy()
        t = now_fn()
        for j, k in enumerate(ks):
            r = self.req[k]
            self.R[:, k] = Rt[:, j]
            self.it[k] = 0
            if rn[j] <= r.tol or r.iters >= r.max_iter:
                r.relres = float(rn[j])
                r.converged = bool(rn[j] <= r.tol)
                r.x = self.X[:, k].clone()
                self._release(k, t, out)


class Server:
    """Resident matrices + continuous batching of matvec / PCG requests."""

    def __init__(self, budget_bytes: float = 150e9, max_slots: int = 16, refresh: int = 200):
        self.budget, self.max_slots, self.refresh = float(budget_bytes), max_slots, refresh
        self.blocks: dict[str, SlotBlock] = {}
        self.footprint: dict[str, float] = {}

    def used_bytes(self) -> float:
        return sum(self.footprint.values())

    def admit_matrix(self, name: str, image: Image, mu: float, precision: str = "mixed") -> bool:
        """Keep the image resident if its footprint (image + slot block) fits the budget."""
        st = image.stats()
        slot_bytes = 8.0 * image.N * self.max_slots * 6
        need = float(st["device_bytes"]) + slot_bytes + 8.0 * image.N * self.max_slots * 4
        if self.used_bytes() + need > self.budget:
            return False
        image.set_precision(precision)
        self.blocks[name] = SlotBlock(ShiftedOperator(image, mu, precision), self.max_slots, self.refresh)
        self.footprint[name] = need
        return True

    def evict(self, name: str):
        self.blocks.pop(name, None)
        self.footprint.pop(name, None)

    def run(self, requests: list[Request], realtime: bool = True) -> list[Request]:
        """Serve requests whose ``arrival`` offsets follow the wall clock (realtime) or
        are all present at time 0 (realtime=False).  Returns them in completion order."""
        pending = [(r.arrival if realtime else 0.0, r.rid, r) for r in requests]
        heapq.heapify(pending)
        waiting: dict[str, list[Request]] = {n: [] for n in self.blocks}
        done: list[Request] = []
        t0 = time.perf_counter()

        def now():
            torch.cuda.synchronize()
            return time.perf_counter() - t0

        while pending or any(waiting.values()) or any(b.busy() for b in self.blocks.values()):
            t = now()
            while pending and pending[0][0] <= t:
                _, _, r = heapq.heappop(pending)
                if r.matrix not in self.blocks:
                    raise KeyError(f"matrix {r.matrix!r} is not resident")
                waiting[r.matrix].append(r)
            for name, blk in self.blocks.items():
                q = waiting[name]
                while q and blk.admit(q[0], t):
                    q.pop(0)
            busy = [b for b in self.blocks.values() if b.busy()]
            if not busy:
                if pending:
                    time.sleep(max(0.0, min(pending[0][0] - now(), 0.001)))
                continue
            for blk in busy:
                blk.step(now, done)
        return done


def latency_stats(reqs: list[Request]) -> dict:
    lat = np.array([r.finish - r.arrival for r in reqs])
    span = max(r.finish for r in reqs) - min(r.arrival for r in reqs)
    return {"n": len(reqs), "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "throughput_req_s": len(reqs) / span if span > 0 else None}
