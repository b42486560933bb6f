"""Multi-process paths on CPU: two gloo ranks on 127.0.0.1 exercise the
replica seeding, the instance sharding of a sweep batch and the timing
reductions that bench.py uses for N > 1 GPUs (no GPU needed)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    from brainpy.state_b200 import dist as D
    r, w, _ = D.world_info()
    mine = D.shard_instances(costs, r, w)
    shards = [None] * w
    dist.all_gather_object(shards, mine)
    t_max = D.max_over_ranks(10.0 + r)
    n_sum = D.sum_over_ranks(len(mine))
    out.put((r, shards, t_max, n_sum, D.replica_seed(1234, r)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    from brainpy.state_b200 import brunel
    specs = brunel.sweep_instances(n=37, seed=3)
    costs = [s["NE"] ** 2 for s in specs]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shards = res[0][1]
    assert shards == res[1][1]                     # every rank sees the same partition
    flat = sorted(shards[0] + shards[1])
    assert flat == list(range(len(specs)))         # disjoint and complete
    load = [sum(costs[i] for i in sh) for sh in shards]
    assert max(load) <= 1.25 * min(load)          # balanced by cost
    assert res[0][2] == res[1][2] == 11.0         # slowest rank's time
    assert res[0][3] == res[1][3] == len(specs)
    assert (res[0][4], res[1][4]) == (1234, 1235)  # independent replicas


def test_single_process_reductions_are_identity():
    from brainpy.state_b200 import dist as D
    assert D.max_over_ranks(3.5) == 3.5
    assert D.sum_over_ranks(2) == 2.0
    assert D.shard_instances([1, 2, 3], 0, 1) == [0, 1, 2]


def _dp_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    import numpy as np
    from brainpy.state_b200 import dist as D
    from brainpy.state_b200.lif_task import make_task
    from oracle import oracle as o
    T = make_task(n_exc=40, n_inh=10, n_in=20, batch=5, n_steps=80, relaxed=True,
                  params=[-70.0, 250.0, 10.0, 0.0, -55.0, -70.0, 2.0, 2.0, 0.0],
                  w_in_scale=900.0, seed=3)
    lo, hi = D.batch_slice(T["cfg"]["batch"], rank, world)
    cfg = dict(T["cfg"], batch=hi - lo)
    loss, dw, dwi, _ = o.lif_bptt(cfg, T["row_ptr"], T["col"], T["w"], T["w_in"],
                                  np.ascontiguousarray(T["inputs"][:, lo:hi]),
                                  np.ascontiguousarray(T["targets"][:, lo:hi]))
    ts = [torch.tensor([loss], dtype=torch.float64), torch.from_numpy(dw.copy()),
          torch.from_numpy(dwi.copy())]
    D.allreduce_mean_grads(ts, hi - lo, T["cfg"]["batch"])
    out.put((rank, (lo, hi), float(ts[0][0]), ts[1].numpy(), ts[2].numpy()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_data_parallel_gradient_equals_full_batch(oracle):
    """Data-parallel BPTT: each rank takes a contiguous share of an odd batch
    (3 + 2 trials), the weighted all-reduce of the per-rank gradients of the
    mean loss gives the full-batch loss and gradient (the oracle is the
    checker for both)."""
    import numpy as np
    from brainpy.state_b200.lif_task import make_task
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [(0, 3), (3, 5)]
    T = make_task(n_exc=40, n_inh=10, n_in=20, batch=5, n_steps=80, relaxed=True,
                  params=[-70.0, 250.0, 10.0, 0.0, -55.0, -70.0, 2.0, 2.0, 0.0],
                  w_in_scale=900.0, seed=3)
    loss, dw, dwi, _ = oracle.lif_bptt(T["cfg"], T["row_ptr"], T["col"], T["w"], T["w_in"],
                                       T["inputs"], T["targets"])
    for r in res:
        assert r[2] == pytest.approx(loss, rel=1e-12)
        np.testing.assert_allclose(r[3], dw, rtol=1e-11, atol=1e-14 * np.abs(dw).max())
        np.testing.assert_allclose(r[4], dwi.reshape(r[4].shape), rtol=1e-11,
                                   atol=1e-14 * np.abs(dwi).max())
    np.testing.assert_array_equal(res[0][3], res[1][3])  # every rank holds the same gradient
