"""The continuous-batching solve server (hg_server_*).

- A served request gives the same solution as the same solve made directly through the
  storage / operator / multigrid API (same seeded right-hand side): 1e-12 relative.
- A request gives the same solution alone and in a mix of concurrent requests of other shapes
  and coefficients that arrive while it runs: 1e-12 relative (the kernels are deterministic, so
  the results are in fact identical).
- Every request of a mix reaches its tolerance; the admission respects the HBM budget (a small
  budget serialises the requests and evicts idle hierarchies; a request larger than the budget
  fails with an error instead of running).
- Admission: requests of a shape whose resident hierarchy is busy wait for it instead of
  building another, and a request of another shape behind them starts first.
- Batched solves: requests queued behind a busy worker are solved together in one union
  hierarchy (disjoint copies of their shape in one storage, one launch per kernel for all of
  them, the coarse-grid CG one block per copy); each gets the iterations, residual and solution
  of its direct solve bit for bit."""
import numpy as np
import pytest

import hyteg_b200 as hg

pytestmark = pytest.mark.gpu
TOL = 1e-8


@pytest.fixture(scope="module")
def gpu():
    if hg.device_count() == 0:
        pytest.skip("no CUDA device")


def direct_solve(k, L, coefficient, seed, dtype):
    st = hg.PrimitiveStorage.cuboid((0, 0, 0), (1, 1, 1), k, k, k, L)
    st.set_cell_coefficients(np.full(6 * k ** 3, coefficient))
    A = hg.P1ConstantLaplaceOperator(st, 0, L)
    x, b = hg.P1Function("x", st, 0, L), hg.P1Function("b", st, 0, L)
    b.fill_random(seed, L, hg.Inner)
    gmg = hg.GeometricMultigridSolver(st, hg.SORSmoother(1.0), hg.CGSolver(st, 0, 0, 200, 1e-16),
                                      hg.P1toP1LinearRestriction(), hg.P1toP1LinearProlongation(), 0, L, 3, 3,
                                      dtype=dtype)
    it, rel, _ = gmg.solve_to(A, x, b, L, TOL, 100)
    _, owned = st.host().slot_info(L)
    return x.to_numpy(L), it, rel, owned


def rel_diff(a, b, owned):
    m = owned == 1
    return np.abs(a[m] - b[m]).max() / np.abs(b[m]).max()


@pytest.mark.parametrize("precision,dtype", [(4, np.float32), (8, np.float64)])
def test_served_request_equals_direct_solve(gpu, precision, dtype):
    k, L, c, seed = 2, 4, 2.5, 7
    ref, it_ref, rel_ref, owned = direct_solve(k, L, c, seed, dtype)
    srv = hg.SolveServer(workers=2, precision=precision)
    rid = srv.submit(k, L, c, seed, TOL, keep_solution=True)
    assert srv.wait(rid, 120.0)
    res = srv.result(rid)
    assert res["status"] == 2 and res["rel_residual"] <= TOL and res["iterations"] == it_ref
    assert res["inner_dofs"] == (k * 2 ** L - 1) ** 3
    assert rel_diff(srv.solution(rid), ref, owned) < 1e-12
    srv.close()


def test_alone_and_in_the_mix_agree(gpu):
    probe = dict(k=2, level=5, coefficient=0.37, seed=11)
    srv = hg.SolveServer(workers=6, precision=4)
    alone = srv.submit(tol=TOL, keep_solution=True, **probe)
    assert srv.wait(alone, 300.0)
    sol_alone = srv.solution(alone)
    rng = np.random.default_rng(5)
    ids = []
    for i in range(14):  # other shapes and coefficients, submitted while the probe runs
        ids.append(srv.submit(int(rng.integers(1, 4)), int(rng.integers(3, 6)), float(np.exp(rng.uniform(-2.3, 2.3))),
                              100 + i, TOL))
        if i == 3:
            mixed = srv.submit(tol=TOL, keep_solution=True, **probe)
    for rid in ids + [mixed]:
        assert srv.wait(rid, 300.0)
        r = srv.result(rid)
        assert r["status"] == 2 and r["rel_residual"] <= TOL
    # the probe overlapped with others (its run interval intersects another request's)
    rm = srv.result(mixed)
    others = [srv.result(i) for i in ids]
    assert any(o["t_start"] < rm["t_end"] and o["t_end"] > rm["t_start"] for o in others)
    _, owned = hg.HostMesh.cuboid((0, 0, 0), (1, 1, 1), 2, 2, 2, 5).slot_info(5)
    assert rel_diff(srv.solution(mixed), sol_alone, owned) < 1e-12
    st = srv.stats()
    assert st["completed"] == 16 and st["failed"] == 0
    srv.close()


def test_budget_admission(gpu):
    # a budget for about one level-5 hierarchy of the 2x2x2 cube: requests run one at a time,
    # hierarchies of other shapes are evicted, and a request that can never fit fails
    srv = hg.SolveServer(workers=4, hbm_budget_bytes=1 << 28, precision=4)
    ids = [srv.submit(k, L, 1.0, s, TOL) for s, (k, L) in enumerate([(1, 4), (2, 5), (1, 3), (2, 4), (1, 5)])]
    for rid in ids:
        assert srv.wait(rid, 300.0)
        assert srv.result(rid)["status"] == 2
    st = srv.stats()
    assert st["peak_bytes"] <= 1 << 28 and st["completed"] == 5
    big = srv.submit(4, 7, 1.0, 0, TOL)
    assert srv.wait(big, 60.0)
    with pytest.raises(hg.HygError):
        srv.result(big)
    srv.close()


@pytest.mark.parametrize("precision,dtype", [(4, np.float32), (8, np.float64)])
def test_batched_requests_equal_direct_solves(gpu, precision, dtype):
    k, L = 2, 4
    reqs = [(0.3, 5), (2.5, 7), (1.0, 9), (7.0, 11), (0.12, 13)]
    srv = hg.SolveServer(workers=1, precision=precision)
    srv.prewarm_batch(k, L, 4)
    srv.set_batching(L)
    busy = srv.submit(3, 5, 1.0, 1, TOL)  # the single worker builds and solves this one meanwhile
    ids = [srv.submit(k, L, c, sd, TOL, keep_solution=True) for c, sd in reqs]
    for i in [busy] + ids:
        assert srv.wait(i, 300.0)
    sizes = []
    for (c, sd), rid in zip(reqs, ids):
        res = srv.result(rid)
        ref, it_ref, rel_ref, owned = direct_solve(k, L, c, sd, dtype)
        assert res["status"] == 2 and res["rel_residual"] <= TOL
        assert res["iterations"] == it_ref
        assert res["rel_residual"] == rel_ref
        assert rel_diff(srv.solution(rid), ref, owned) == 0.0
        sizes.append(res["batch_size"])
    assert sizes[:4] == [4, 4, 4, 4] and sizes[4] == 1, sizes
    srv.close()


def test_busy_shape_waits_and_other_shapes_pass(gpu):
    srv = hg.SolveServer(workers=2, precision=4)
    srv.prewarm(2, 6)
    srv.prewarm(1, 3)
    first = srv.submit(2, 6, 1.0, 1, TOL)            # takes the one (2, 6) hierarchy
    waiting = [srv.submit(2, 6, 1.0 + i, 2 + i, TOL) for i in range(3)]
    other = srv.submit(1, 3, 1.0, 9, TOL)            # behind them in the queue, another shape
    for rid in [first] + waiting + [other]:
        assert srv.wait(rid, 300.0)
    res = {rid: srv.result(rid) for rid in [first] + waiting + [other]}
    assert not any(r["built_hierarchy"] for r in res.values())  # nothing was built on admission
    # the (2, 6) requests ran one after another on their hierarchy ...
    runs = sorted((res[r]["t_start"], res[r]["t_end"]) for r in [first] + waiting)
    assert all(a[1] <= b[0] for a, b in zip(runs, runs[1:]))
    # ... and the later request of another shape did not wait for them
    assert res[other]["t_start"] < max(res[r]["t_start"] for r in waiting)
    st = srv.stats()
    assert st["completed"] == 5 and st["failed"] == 0
    srv.close()
