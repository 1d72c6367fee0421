"""Host logic of the multi-GPU path: independent operators split across ranks
(gloo, world size 2, on CPU), results gathered in the original order."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import __graft_entry__ as ge

ek = ge.load_package()
from edkit_b200.sharding import partition, sharded_solve  # noqa: E402


def test_partition_balances_uneven_weights():
    rng = np.random.default_rng(0)
    dims = [924, 3432, 12870, 48620, 184756]
    w = [dims[i] for i in rng.integers(0, 5, 512)]
    parts = partition(w, 4)
    assert sorted(i for p in parts for i in p) == list(range(512))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)
    assert partition(w, 4) == parts  # deterministic


def test_partition_edge_cases():
    assert partition([], 3) == [[], [], []]
    assert partition([5.0], 2) == [[0], []]
    assert partition([1, 1, 1], 1) == [[0, 1, 2]]
    with pytest.raises(ValueError):
        partition([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, specs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        built = []

        def build(s):
            built.append(s)
            return s

        def solve(ops):  # stands in for batch_lanczos_e0: two "levels" per problem
            return np.array([[-s[0] * s[1], s[0] + 0.5] for s in ops])

        res, mine = sharded_solve(specs, build, solve, weight=lambda s: s[0] ** 2)
        q.put((rank, res.tolist(), mine, [list(b) for b in built]))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_restores_order():
    specs = [(L, k) for L in (12, 14, 16, 20, 26) for k in range(3)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, specs, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = np.array([[-L * k, L + 0.5] for L, k in specs])
    mines = {}
    for rank, res, mine, built in out:
        assert np.array_equal(np.array(res), want)
        assert [tuple(b) for b in built] == [specs[i] for i in mine]  # built only its share
        mines[rank] = mine
    assert sorted(mines[0] + mines[1]) == list(range(len(specs)))
    assert not set(mines[0]) & set(mines[1])


def test_single_process_runs_everything():
    specs = [(3, 1), (5, 2)]
    res, mine = sharded_solve(specs, lambda s: s, lambda ops: [[a * b] for a, b in ops])
    assert mine == [0, 1] and np.array_equal(res, [[3], [10]])


def _chain_spec(q):
    """A small random-field XXZ chain (open, N = L/2), as in the disorder ensemble."""
    rng = np.random.default_rng(100 + q)
    L = int(rng.choice([8, 10]))
    return (q, L, [float(h) for h in rng.uniform(-3, 3, L)])


def _oracle_low2(spec):
    """The two lowest levels of a chain from the oracle's dense matrix."""
    import oracle as O
    _, L, h = spec
    inds = [[i, i + 1] for i in range(1, L)] + [[i] for i in range(1, L + 1)]
    mats = [O.spin((1.0, "xx"), (1.0, "yy"), (1.0, "zz"))] * (L - 1) + [hi * O.spin("z") for hi in h]
    Ho = O.operator(mats, inds, O.projected(L, N=L // 2))
    return np.linalg.eigvalsh(Ho.dense())[:2]


def _eig_worker(rank, world, port, specs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from math import comb
        res, mine = sharded_solve(specs, lambda s: s,
                                  lambda ops: np.array([_oracle_low2(s) for s in ops]),
                                  weight=lambda s: comb(s[1], s[1] // 2) * s[1])
        q.put((rank, res.tolist(), mine))
    finally:
        dist.destroy_process_group()


def test_two_rank_ensemble_eigenvalues_match_a_single_process():
    """Real eigenvalues through the sharded path: twelve disorder instances
    split over two gloo ranks, each rank solving its share (the oracle's
    dense spectra standing in for the GPU solver on this CPU-only test), give
    exactly the single-process results in the original order."""
    specs = [_chain_spec(q) for q in range(12)]
    want = np.array([_oracle_low2(s) for s in specs])
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_eig_worker, args=(r, 2, port, specs, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mines = []
    for rank, res, mine in out:
        assert np.array_equal(np.array(res), want)
        mines.append(mine)
    assert mines[0] and mines[1] and sorted(mines[0] + mines[1]) == list(range(12))
