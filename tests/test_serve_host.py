"""Host logic of the served form (h2pack_b200/serve.py) with a stand-in CG engine: no GPU.

The stand-in SlotBlock finishes a request once it has run ``max_iter`` iterations
(``iters_per_sync`` per launch).  It records what the scheduler asked of it.  The
tests check:

- the HBM budget admits or refuses resident matrices;
- requests of one matrix queue FIFO behind its 16 (here 2) slots;
- a finished request frees its slot for the next one at once;
- every busy engine is launched before any is collected, so their device work
  overlaps;
- engines are decoupled: a fast engine's requests finish while a slow engine's
  iterations are still in flight (no head-of-line blocking across matrices);
- a request past its deadline leaves its queue or its slot (cancelled) with status
  "timeout", and its slot serves the next request;
- an unknown matrix is an error.
"""
import pytest

from h2pack_b200 import serve


class FakeImage:
    def __init__(self, N, device_bytes, latency=0):
        self.N = N
        self._bytes = device_bytes
        self.lib = None
        self.latency = latency

    def stats(self):
        return {"device_bytes": self._bytes}


class FakeBlock:
    log = []   # ("launch" | "collect", matrix id) in call order, shared by all blocks

    def __init__(self, image, mu, precision, max_slots, refresh, iters_per_sync):
        self.img, self.S, self.k = image, max_slots, iters_per_sync
        self.free = list(range(max_slots))[::-1]
        self.req = {}
        self.done_iters = {}
        self.history = False
        self.max_in_flight = 0
        self.inflight = False
        self.polls_left = 0
        self.cancelled = []
        self.latency = getattr(image, "latency", 0)   # polls until a launch is done

    def busy(self):
        return len(self.free) < self.S

    def admit(self, r, now):
        if not self.free:
            return False
        k = self.free.pop()
        self.req[k] = r
        self.done_iters[k] = 0
        r.start = now
        self.max_in_flight = max(self.max_in_flight, len(self.req))
        return True

    def launch(self):
        FakeBlock.log.append(("launch", id(self)))
        for k in self.req:
            self.done_iters[k] += self.k
        self.inflight = True
        self.polls_left = self.latency

    def ready(self):
        if self.polls_left > 0:
            self.polls_left -= 1
            return False
        return True

    def requests(self):
        return list(self.req.values())

    def cancel(self, r):
        for k, q in list(self.req.items()):
            if q is r:
                del self.req[k]
                self.free.append(k)
                self.cancelled.append(r.rid)
                return True
        return False

    def collect(self, now_fn, out):
        FakeBlock.log.append(("collect", id(self)))
        self.inflight = False
        t = now_fn()
        for k in sorted(self.req):
            r = self.req[k]
            if self.done_iters[k] >= r.max_iter:
                r.iters, r.finish, r.converged, r.relres, r.status = self.done_iters[k], t, True, 0.0, "done"
                out.append(r)
                del self.req[k]
                self.free.append(k)

    def close(self):
        pass


@pytest.fixture
def fake_engine(monkeypatch):
    class _Stream:
        def synchronize(self):
            pass
    monkeypatch.setattr(serve, "SlotBlock", FakeBlock)
    monkeypatch.setattr(serve.torch.cuda, "current_stream", lambda: _Stream())
    FakeBlock.log = []
    return FakeBlock


def req(rid, matrix, iters, kind="pcg", timeout=None):
    return serve.Request(rid=rid, matrix=matrix, kind=kind, b=None, max_iter=iters, timeout=timeout)


def test_budget_admits_and_refuses(fake_engine):
    N = 10
    engine = 8.0 * N * 16 * 5
    srv = serve.Server(budget_bytes=2 * (1000 + engine) + 1)
    assert srv.admit_matrix("a", FakeImage(N, 1000), mu=1e-2)
    assert srv.admit_matrix("b", FakeImage(N, 1000), mu=1e-2)
    assert not srv.admit_matrix("c", FakeImage(N, 1000), mu=1e-2)
    assert srv.used_bytes() == pytest.approx(2 * (1000 + engine))
    srv.evict("a")
    assert srv.admit_matrix("c", FakeImage(N, 1000), mu=1e-2)


def test_fifo_queue_and_slot_reuse(fake_engine):
    srv = serve.Server(budget_bytes=1e12, max_slots=2, iters_per_sync=8)
    assert srv.admit_matrix("m", FakeImage(4, 0), mu=1e-2)
    rs = [req(0, "m", 8), req(1, "m", 8), req(2, "m", 16), req(3, "m", 8), req(4, "m", 8)]
    done = srv.run(rs, realtime=False)
    assert sorted(r.rid for r in done) == [0, 1, 2, 3, 4]
    order = [r.rid for r in done]
    # 0 and 1 take the two slots and finish in the first batch; 2 and 3 enter next,
    # 3 finishes first and hands its slot to 4; 2 needs a second batch
    assert set(order[:2]) == {0, 1}
    assert order.index(3) < order.index(2)
    assert order.index(3) < order.index(4)
    assert srv.blocks["m"].max_in_flight == 2
    assert all(r.iters >= r.max_iter and r.converged for r in done)
    assert len([e for e in FakeBlock.log if e[0] == "launch"]) == 3


def test_engines_of_different_matrices_overlap(fake_engine):
    srv = serve.Server(budget_bytes=1e12, max_slots=4, iters_per_sync=8)
    assert srv.admit_matrix("a", FakeImage(4, 0), mu=1e-2)
    assert srv.admit_matrix("b", FakeImage(4, 0), mu=1e-2)
    done = srv.run([req(0, "a", 16), req(1, "b", 16), req(2, "a", 8, kind="matvec")], realtime=False)
    assert sorted(r.rid for r in done) == [0, 1, 2]
    # each scheduling round launches every busy engine before collecting any
    log = [e[0] for e in FakeBlock.log]
    assert log[:4] == ["launch", "launch", "collect", "collect"]


def test_unknown_matrix_is_an_error(fake_engine):
    srv = serve.Server(budget_bytes=1e12)
    assert srv.admit_matrix("a", FakeImage(4, 0), mu=1e-2)
    with pytest.raises(KeyError):
        srv.run([req(0, "nope", 8)], realtime=False)


def test_fast_engine_does_not_wait_for_a_slow_one(fake_engine):
    """A slow engine (its launches take 200 polls) and a fast one: every request of the
    fast matrix finishes while the slow engine's first launch is still in flight."""
    srv = serve.Server(budget_bytes=1e12, max_slots=2, iters_per_sync=8)
    assert srv.admit_matrix("slow", FakeImage(4, 0, latency=200), mu=1e-2)
    assert srv.admit_matrix("fast", FakeImage(4, 0), mu=1e-2)
    reqs = [req(0, "slow", 8)] + [req(1 + i, "fast", 16) for i in range(6)]
    done = srv.run(reqs, realtime=False, poll_sleep=0.0)
    order = [r.rid for r in done]
    assert order[-1] == 0                     # the slow request finishes last ...
    assert sorted(order[:-1]) == list(range(1, 7))
    slow = srv.blocks["slow"]
    collects = [i for i, e in enumerate(FakeBlock.log) if e == ("collect", id(slow))]
    fast_collects = [i for i, e in enumerate(FakeBlock.log) if e[0] == "collect" and e[1] != id(slow)]
    assert len(collects) == 1                 # ... after one launch of its own,
    assert len(fast_collects) >= 6 and max(fast_collects) < collects[0]   # which the fast engine never waited for


def test_requests_past_their_deadline_time_out(fake_engine):
    """One slot: the first request holds it past its deadline and is cancelled; the
    queued request behind it with a short deadline expires in the queue; the third
    (no deadline) then runs to completion in the freed slot."""
    srv = serve.Server(budget_bytes=1e12, max_slots=1, iters_per_sync=8)
    assert srv.admit_matrix("m", FakeImage(4, 0, latency=10 ** 9), mu=1e-2)
    blk = srv.blocks["m"]
    reqs = [req(0, "m", 8, timeout=0.02), req(1, "m", 8, timeout=0.01), req(2, "m", 8)]

    # the slot's first launch never finishes on its own; once request 0 is cancelled the
    # engine is made fast so that request 2 can complete
    orig_cancel = blk.cancel

    def cancel(r):
        ok = orig_cancel(r)
        blk.latency = 0
        blk.polls_left = 0
        return ok
    blk.cancel = cancel
    done = srv.run(reqs, realtime=False, poll_sleep=0.0)
    st = {r.rid: r.status for r in done}
    assert st == {0: "timeout", 1: "timeout", 2: "done"}
    assert blk.cancelled == [0]
    stats = serve.latency_stats(done)
    assert stats["n"] == 1 and stats["n_timeout"] == 2
