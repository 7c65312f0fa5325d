"""Served form: resident matrices, continuous batching of matvec and PCG requests on
(K + mu I), admission by device footprint, and the same result alone and in the mix."""
import numpy as np
import pytest

from conftest import make_points, rel

pytestmark = pytest.mark.gpu
MU = 1e-2


def build(kernel, n, seed, ell):
    from h2pack_b200 import H2Matrix
    param = [1.0 / ell ** 2] if kernel == "gaussian" else [1.0 / ell]
    return H2Matrix(kernel, make_points(kernel, n, seed), param, 1e-6, BD_JIT=1, max_leaf_points=200)


@pytest.fixture(scope="module")
def mats():
    Hs = {"g": build("gaussian", 6000, 1, 1.0), "m": build("matern32", 4000, 2, 0.7)}
    yield Hs
    for H in Hs.values():
        H.close()


def fp64_apply(H, x):
    import torch
    img = H.image()
    img.set_precision("fp64")
    y = img.matmul_device(x.reshape(-1, 1).contiguous())[:, 0]
    return y + MU * x


def requests(H, kinds, seed, name):
    import torch
    from h2pack_b200.serve import Request
    g = torch.Generator(device="cuda").manual_seed(seed)
    return [Request(rid=seed * 100 + i, matrix=name, kind=k,
                    b=torch.randn(H.N, dtype=torch.float64, device="cuda", generator=g)) for i, k in enumerate(kinds)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pcg_converges_to_tolerance(mats, precision):
    import torch
    from h2pack_b200.serve import Server
    H = mats["g"]
    srv = Server(max_slots=4)
    assert srv.admit_matrix("g", H.image(), MU, precision)
    reqs = requests(H, ["pcg", "pcg"], 3, "g")
    done = srv.run(reqs, realtime=False)
    assert len(done) == 2
    for r in done:
        assert r.converged and r.relres <= 1e-6
        res = torch.linalg.vector_norm(r.b - fp64_apply(H, r.x)) / torch.linalg.vector_norm(r.b)
        assert float(res) <= 1.5e-6


def test_matvec_request_is_shifted_apply(mats):
    from h2pack_b200.serve import Server
    H = mats["m"]
    srv = Server(max_slots=4)
    assert srv.admit_matrix("m", H.image(), MU, "fp64")
    (r,) = requests(H, ["matvec"], 4, "m")
    (d,) = srv.run([r], realtime=False)
    assert rel(d.x.cpu().numpy(), fp64_apply(H, r.b).cpu().numpy()) < 1e-13


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_same_result_alone_and_in_the_mix(mats, precision):
    """A request's answer does not depend on what else is being served."""
    from h2pack_b200.serve import Server
    Hg, Hm = mats["g"], mats["m"]
    probe_pcg = requests(Hg, ["pcg"], 7, "g")[0]
    probe_mv = requests(Hm, ["matvec"], 8, "m")[0]

    def serve(reqs):
        srv = Server(max_slots=8)
        assert srv.admit_matrix("g", Hg.image(), MU, precision)
        assert srv.admit_matrix("m", Hm.image(), MU, precision)
        return {r.rid: r for r in srv.run(reqs, realtime=True)}

    import copy
    alone = serve([copy.copy(probe_pcg), copy.copy(probe_mv)])
    mix = requests(Hg, ["pcg", "matvec", "pcg", "pcg", "matvec"], 9, "g") + \
        requests(Hm, ["pcg", "matvec", "pcg"], 10, "m")
    for i, r in enumerate(mix):
        r.arrival = 0.002 * i          # arrivals while others are already on the GPU
    a, b = copy.copy(probe_pcg), copy.copy(probe_mv)
    a.arrival, b.arrival = 0.003, 0.005
    mixed = serve(mix + [a, b])
    xa, xm = alone[probe_pcg.rid].x.cpu().numpy(), mixed[probe_pcg.rid].x.cpu().numpy()
    tol_sol = 1e-12 if precision == "fp64" else 2e-4
    assert mixed[probe_pcg.rid].relres <= 1e-6 and alone[probe_pcg.rid].relres <= 1e-6
    assert rel(xm, xa) < max(tol_sol, 1e-4)
    tol_mv = 1e-13 if precision == "fp64" else 2e-6
    assert rel(mixed[probe_mv.rid].x.cpu().numpy(), alone[probe_mv.rid].x.cpu().numpy()) < tol_mv


def test_admission_by_footprint(mats):
    from h2pack_b200.serve import Server
    H = mats["g"]
    img = H.image()
    need = img.stats()["device_bytes"]
    srv = Server(budget_bytes=need * 0.5, max_slots=4)
    assert not srv.admit_matrix("g", img, MU)
    srv = Server(budget_bytes=need * 10 + 1e8, max_slots=4)
    assert srv.admit_matrix("g", img, MU)
    assert not srv.admit_matrix("g2", img, MU) or srv.used_bytes() <= srv.budget


def test_pcg_fp64_follows_reference_pcg(mats):
    """The served solver with the FP64 operator against pcg.c restated (oracle.pcg) driven by
    the reference library's own CPU H2P_matvec on the same handle: the residual histories
    agree while rounding differences are still small, and both converge in nearly the same
    number of iterations."""
    import torch
    from oracle import oracle as O
    from h2pack_b200.serve import Server, Request
    H = mats["m"]
    g = torch.Generator(device="cuda").manual_seed(21)
    b = torch.randn(H.N, dtype=torch.float64, device="cuda", generator=g)
    srv = Server(max_slots=2)
    assert srv.admit_matrix("m", H.image(), MU, "fp64")
    done = srv.run([Request(rid=1, matrix="m", kind="pcg", b=b, tol=1e-6)], realtime=False, history=True)
    r = done[0]

    def cpu_apply(x):
        y = np.zeros_like(x)
        O.libref().H2P_matvec(H.h2pack, O.dptr(np.ascontiguousarray(x)), O.dptr(y))
        return y + MU * x

    bh = b.cpu().numpy()
    x, flag, relres, iters, hist = O.pcg(cpu_apply, bh, 1e-6, 5000)
    assert flag == 0 and r.converged
    assert abs(r.iters - iters) <= max(3, iters // 20)
    h_gpu = np.array(r.history)
    k = min(20, len(hist), len(h_gpu))
    assert np.max(np.abs(h_gpu[:k] - hist[:k]) / hist[:k]) < 1e-8
    assert rel(r.x.cpu().numpy(), x) < 1e-3


def test_deadline_cancels_a_slot_and_frees_it(mats):
    """One slot: a PCG request with a tiny deadline is cancelled on the device after its
    first launch; the matvec queued behind it then takes the freed slot and gives the
    exact shifted product."""
    from h2pack_b200.serve import Server
    H = mats["g"]
    srv = Server(max_slots=1)
    assert srv.admit_matrix("g", H.image(), MU, "fp64")
    slow, mv = requests(H, ["pcg", "matvec"], 11, "g")
    slow.timeout, slow.tol = 1e-4, 1e-14        # cannot finish in time
    done = {r.rid: r for r in srv.run([slow, mv], realtime=False)}
    assert done[slow.rid].status == "timeout" and done[slow.rid].x is None
    assert done[mv.rid].status == "done"
    assert rel(done[mv.rid].x.cpu().numpy(), fp64_apply(H, mv.b).cpu().numpy()) < 1e-13
