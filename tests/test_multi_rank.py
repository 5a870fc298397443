"""Multi-rank path on CPU: two gloo ranks shard a batch of scenarios, each
differentiates its block (oracle), and the batch-summed roughness and emitter
gradients are all-reduced.  The result must equal the single-process full
batch."""
import os
import socket

import numpy as np
import pytest

from wdsgpu_b200.sharding import scenario_shard


def test_shards_cover_the_batch_once():
    for n in (0, 1, 5, 1024, 1023):
        for world in (1, 2, 3, 8):
            got = [scenario_shard(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        scenario_shard(4, 2, 2)


def _inputs():
    from wdsgpu_b200 import synth
    net = synth.feature_network()
    d, _ = synth.config2_scenarios(net, 5, seed=21, sigma=0.3)
    rh = np.broadcast_to(net.fixed_head_ft_at(0), d.shape).copy()
    return net, d, rh, synth.sensor_nodes(net, 6)


def _grads(net, d, rh, sens):
    from oracle.gga import Model
    m = Model(net)
    out, st = m.implicit(d, rh, accuracy=1e-7, polish_steps=3)
    gH = np.zeros_like(out["head_ft"])
    gH[:, sens] = 2.0 * out["head_ft"][:, sens]
    gd, grh, gke, gr = m.backward(st, gH, np.zeros_like(out["flow_cfs"]),
                                  np.zeros_like(out["emitter_cfs"]))
    return gr.sum(0), gke.sum(0), gd


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from wdsgpu_b200.sharding import allreduce_batch_summed
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        net, d, rh, sens = _inputs()
        lo, hi = scenario_shard(d.shape[0], rank, world)
        gr, gke, gd = _grads(net, d[lo:hi], rh[lo:hi], sens)
        tr, tk = torch.tensor(gr), torch.tensor(gke)
        allreduce_batch_summed([tr, tk])
        q.put((rank, lo, hi, tr.numpy(), tk.numpy(), gd))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_full_batch_gradient():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    net, d, rh, sens = _inputs()
    gr, gke, gd = _grads(net, d, rh, sens)
    for rank, lo, hi, tr, tk, gdr in res:
        np.testing.assert_allclose(tr, gr, rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(tk, gke, rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(gdr, gd[lo:hi], rtol=1e-10, atol=1e-14)
