"""Batched solves: many independent uneven SPD systems in one persistent
launch, checked system by system against the FP64 oracle."""
import numpy as np
import pytest

from seldon_b200 import matgen
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api(cuda):
    from seldon_b200 import api
    return api


def _systems(seed, k, lo, hi, zero=()):
    rng = np.random.default_rng(seed)
    systems, rhs, xs = [], [], []
    for s in range(k):
        g = int(rng.integers(lo, hi + 1))
        ptr, ind, val = matgen.lap2d(g, shift=0.01)
        x = rng.uniform(-1, 1, g * g)
        systems.append((ptr, ind, val))
        xs.append(x)
        rhs.append(np.zeros(g * g) if s in zero else matgen.matvec(ptr, ind, val, x))
    return systems, rhs, xs


PLANS = [(128, 0), (256, 0), (512, 0), (256, 64), (512, 1024), (128, 100000)]


@pytest.mark.parametrize("mixed", [True, False])
@pytest.mark.parametrize("plan", PLANS)
def test_batch_matches_oracle(api, oracle, mixed, plan):
    """Every plan: CTAs only, warps for the smaller systems, warps for all."""
    systems, rhs, xs = _systems(1, 40, 4, 30)
    B = api.Batch(systems)
    B.set_plan(*plan)
    assert B.plan() == plan
    import torch
    X = torch.zeros(B.m, dtype=torch.float64, device="cuda")
    it = torch.zeros(B.nsys, dtype=torch.int32, device="cuda")
    rr = torch.zeros(B.nsys, dtype=torch.float64, device="cuda")
    res = B.solve(X, to_dev(np.concatenate(rhs)), it, rr, tol=1e-9, mixed=mixed)
    assert res.converged == B.nsys and res.max_rel_residual < 1e-9
    x = to_host(X)
    its = to_host(it)
    for s, ((ptr, ind, val), b) in enumerate(zip(systems, rhs)):
        xsys = x[B.sys_row[s]:B.sys_row[s + 1]]
        rel = np.linalg.norm(b - matgen.matvec(ptr, ind, val, xsys)) / np.linalg.norm(b)
        assert rel < 1e-9, (s, rel)
        xo, co, no, _, _ = oracle.solve("cg", ptr, ind, val, b, tol=1e-9, max_iter=2000)
        assert np.linalg.norm(xsys - xo) / np.linalg.norm(xo) < 1e-6
        if not mixed:
            assert abs(int(its[s]) - no) <= max(2, no // 20), (s, its[s], no)


# cluster plans: (threads, warp_max, CTAs per cluster, systems above this
# many rows take a whole cluster)
CLUSTER_PLANS = [(512, 256, 4, 200), (256, 0, 2, 0), (128, 64, 8, 400), (512, 0, 8, 0)]


@pytest.mark.parametrize("mixed", [True, False])
@pytest.mark.parametrize("plan", CLUSTER_PLANS)
def test_batch_cluster_plans_match_oracle(api, oracle, mixed, plan):
    """The largest systems solved by whole thread-block clusters (rows
    spread over the CTAs, sums through distributed shared memory), the rest
    by CTAs and warps: every system against the oracle, repeat solves bit
    for bit."""
    import torch
    systems, rhs, xs = _systems(5, 40, 4, 36)
    B = api.Batch(systems)
    B.set_plan(*plan)
    assert B.plan() == plan[:2] and B.cluster_plan() == plan[2:]
    b = to_dev(np.concatenate(rhs))
    X = torch.zeros(B.m, dtype=torch.float64, device="cuda")
    it = torch.zeros(B.nsys, dtype=torch.int32, device="cuda")
    rr = torch.zeros(B.nsys, dtype=torch.float64, device="cuda")
    res = B.solve(X, b, it, rr, tol=1e-9, mixed=mixed)
    assert res.converged == B.nsys and res.max_rel_residual < 1e-9
    x = to_host(X).copy()
    its = to_host(it)
    for s, ((ptr, ind, val), bb) in enumerate(zip(systems, rhs)):
        xsys = x[B.sys_row[s]:B.sys_row[s + 1]]
        rel = np.linalg.norm(bb - matgen.matvec(ptr, ind, val, xsys)) / np.linalg.norm(bb)
        assert rel < 1e-9, (s, rel)
        xo, co, no, _, _ = oracle.solve("cg", ptr, ind, val, bb, tol=1e-9, max_iter=2000)
        assert np.linalg.norm(xsys - xo) / np.linalg.norm(xo) < 1e-6
        if not mixed:
            assert abs(int(its[s]) - no) <= max(2, no // 20), (s, its[s], no)
    X.zero_()
    B.solve(X, b, it, rr, tol=1e-9, mixed=mixed)
    assert np.array_equal(to_host(X), x)
    # a two-number plan clears the cluster part
    B.set_plan(256, 0)
    assert B.cluster_plan() == (0, 0)


def test_batch_cluster_plan_few_large_systems(api, oracle):
    """Fewer large systems than the GPU's CTA slots: a cluster per system
    against one CTA per system, same answers; timings printed."""
    import time
    import torch
    systems, rhs, xs = _systems(9, 12, 150, 180)
    B = api.Batch(systems)
    b = to_dev(np.concatenate(rhs))
    X = torch.zeros(B.m, dtype=torch.float64, device="cuda")
    it = torch.zeros(B.nsys, dtype=torch.int32, device="cuda")
    rr = torch.zeros(B.nsys, dtype=torch.float64, device="cuda")
    out = {}
    for plan in [(512, 0), (512, 0, 8, 0), (512, 0, 16, 0)]:
        B.set_plan(*plan)
        try:
            B.solve(X, b, it, rr, tol=1e-9)
        except Exception as e:  # a cluster size the GPU cannot schedule
            from seldon_b200._lib import SeldonB200Error
            assert isinstance(e, SeldonB200Error) and plan[2] == 16
            continue
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = B.solve(X, b, it, rr, tol=1e-9)
        out[plan] = (time.perf_counter() - t0) * 1e3
        assert res.converged == B.nsys
        x = to_host(X)
        for s in (0, 5, 11):
            ptr, ind, val = systems[s]
            xsys = x[B.sys_row[s]:B.sys_row[s + 1]]
            xo, _, _, _, _ = oracle.solve("cg", ptr, ind, val, rhs[s], tol=1e-9, max_iter=5000)
            assert np.linalg.norm(xsys - xo) / np.linalg.norm(xo) < 1e-6
    print("few large systems, ms:", {k: round(v, 2) for k, v in out.items()})


def test_batch_cluster_plan_wide_columns(api, oracle):
    """A system of more than 65,536 rows makes the batch keep 4-byte local
    columns; a cluster solves it, CTAs and warps the small ones."""
    import torch
    big = matgen.lap2d(262, shift=0.01)  # 68,644 rows
    systems, rhs, _ = _systems(11, 10, 4, 40)
    xs = np.random.default_rng(12).uniform(-1, 1, 262 * 262)
    systems.insert(3, big)
    rhs.insert(3, matgen.matvec(*big, xs))
    B = api.Batch(systems)
    B.set_plan(512, 256, 8, 1000)
    b = to_dev(np.concatenate(rhs))
    X = torch.zeros(B.m, dtype=torch.float64, device="cuda")
    it = torch.zeros(B.nsys, dtype=torch.int32, device="cuda")
    rr = torch.zeros(B.nsys, dtype=torch.float64, device="cuda")
    res = B.solve(X, b, it, rr, tol=1e-9, max_iter=20000)
    assert res.converged == B.nsys and res.max_rel_residual < 1e-9
    x = to_host(X)
    for s in (0, 3, 10):
        ptr, ind, val = systems[s]
        xsys = x[B.sys_row[s]:B.sys_row[s + 1]]
        xo, _, _, _, _ = oracle.solve("cg", ptr, ind, val, rhs[s], tol=1e-9, max_iter=20000)
        assert np.linalg.norm(xsys - xo) / np.linalg.norm(xo) < 1e-6


def test_batch_edges(api):
    import torch
    systems, rhs, xs = _systems(2, 6, 3, 12, zero=(2,))
    B = api.Batch(systems)
    x0 = np.arange(B.m, dtype=float)
    X = to_dev(x0)
    it = torch.zeros(B.nsys, dtype=torch.int32, device="cuda")
    rr = torch.zeros(B.nsys, dtype=torch.float64, device="cuda")
    res = B.solve(X, to_dev(np.concatenate(rhs)), it, rr, tol=1e-9, init_guess_null=False)
    x = to_host(X)
    # the system with a zero right-hand side is left as it was
    a, e = B.sys_row[2], B.sys_row[3]
    assert np.array_equal(x[a:e], x0[a:e]) and int(to_host(it)[2]) == 0
    assert res.converged == B.nsys
    # entries may not cross systems
    from seldon_b200._lib import SeldonB200Error
    bad = [(np.array([0, 1, 2]), np.array([0, 2]), np.array([1.0, 1.0])),
           (np.array([0, 1]), np.array([0]), np.array([1.0]))]
    with pytest.raises(SeldonB200Error):
        api.Batch(bad)


def test_batch_autotune_and_graph(api):
    import torch
    systems, rhs, xs = _systems(3, 64, 6, 40)
    B = api.Batch(systems)
    b = to_dev(np.concatenate(rhs))
    X = torch.zeros(B.m, dtype=torch.float64, device="cuda")
    assert B.autotune(X, b, tol=1e-9) in (128, 256, 512)
    chosen = B.plan()
    chosen_cluster = B.cluster_plan()
    assert chosen[1] in (0, 256, 1024)
    assert chosen_cluster[0] in (0, 4, 16)
    # a batch with the same size histogram takes the cached plan, cluster part included
    B2 = api.Batch(systems)
    B2.set_plan(128, 0, 2, 5)
    B2.autotune(X, b, tol=1e-9)
    assert B2.plan() == chosen and B2.cluster_plan() == chosen_cluster
    B2.close()
    # the solve enqueues only device work: capture it once, replay it
    X.zero_()
    it = torch.zeros(B.nsys, dtype=torch.int32, device="cuda")
    rr = torch.zeros(B.nsys, dtype=torch.float64, device="cuda")
    B.solve(X, b, it, rr, tol=1e-9)
    ref = to_host(X).copy()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        B.solve(X, b, it, rr, summary=False, tol=1e-9)
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        B.solve(X, b, it, rr, summary=False, tol=1e-9)
    X.fill_(7.0)
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(to_host(X), ref)  # deterministic: same result bit for bit
    assert float(to_host(rr).max()) < 1e-9
