"""Multi-rank reductions (champ_b200.dist) with two gloo ranks on the CPU.

Walkers are sharded across ranks with no data-path exchange; what ranks do exchange are sums:
VMC block estimators, the linear method's O/H accumulators and the DMC weight per step.  Each
test splits one synthetic walker set over two ranks, reduces, and compares with the single-rank
result on all walkers (FP64 sums: equal to rounding).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oh(dl, de, el, wt):
    """S, H as champ_accumulate_oh forms them: Oa = (1, O), Mb = (E_L, E_L O + dE), weighted."""
    Oa = np.hstack([np.ones((len(el), 1)), dl])
    Mb = np.hstack([el[:, None], el[:, None] * dl + de])
    return (wt[:, None] * Oa).T @ Oa, (wt[:, None] * Oa).T @ Mb


def _data(nw=37, P=5, seed=3):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=(nw, P)), rng.normal(size=(nw, P)), rng.normal(-10, 1, nw), rng.uniform(0.5, 1.5, nw),
            rng.normal(-10, 1, nw), rng.uniform(50, 150, nw), rng.uniform(0, 8, nw))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from champ_b200 import dist as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dl, de, el, wt, es, e2, acc = _data()
        lo, n = D.shard(len(el), rank, world)
        sl = slice(lo, lo + n)
        S, H = _oh(dl[sl], de[sl], el[sl], wt[sl])
        Sg, Hg = D.reduce_oh_host(S, H)
        est = D.reduce_estimators(es[sl], e2[sl], acc[sl], nsweep=3, nelec=8)
        mx = D.max_over_ranks(float(rank + 0.5))
        dmc = D.reduce_dmc_step(float(wt[sl].sum()), n, float((wt[sl] * el[sl]).sum()))
        q.put((rank, Sg, Hg, est, mx, dmc))
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out, key=lambda t: t[0])


def test_shard_covers_every_walker_once():
    from champ_b200.dist import shard
    for total in (1, 7, 8192, 4097):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, n = shard(total, r, world)
                seen += list(range(lo, lo + n))
            assert seen == list(range(total))


def test_oh_reduction_equals_single_rank(two_ranks):
    dl, de, el, wt, *_ = _data()
    S, H = _oh(dl, de, el, wt)
    for _, Sg, Hg, *_ in two_ranks:
        assert np.allclose(Sg, S, rtol=1e-13, atol=1e-12)
        assert np.allclose(Hg, H, rtol=1e-13, atol=1e-12)


def test_estimators_max_and_dmc_totals(two_ranks):
    dl, de, el, wt, es, e2, acc = _data()
    n = len(el) * 3
    for _, _, _, est, mx, dmc in two_ranks:
        assert abs(est["energy"] - es.sum() / n) < 1e-12
        assert abs(est["variance"] - (e2.sum() / n - (es.sum() / n) ** 2)) < 1e-9
        assert abs(est["accept"] - acc.sum() / (n * 8)) < 1e-12
        assert est["walkers"] == len(el)
        assert mx == 1.5
        assert abs(dmc[0] - wt.sum()) < 1e-12 and dmc[1] == len(el) and abs(dmc[2] - (wt * el).sum()) < 1e-9
