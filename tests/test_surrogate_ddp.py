"""Data-parallel surrogate training on CPU: world_size 2 over gloo, torch's conv3d standing in for the
tensor-core kernels (the sharding of each global mini-batch, the single gradient all-reduce per step and the
shared normalisation are what is under test). Both ranks must end with the same weights, bit for bit equal to
one process that accumulates the gradients of the same two slices per step."""
import os
import socket

import torch
import torch.multiprocessing as mp

from xadvcool_b200 import surrogate as S
from xadvcool_b200 import warmstart as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _data():
    g = torch.Generator().manual_seed(7)
    feats = torch.rand(4, 8, 16, 24, S.IN_FEATURES, generator=g).to(S.BF16)
    tgts = torch.randn(4, 8, 16, 24, S.OUT_FIELDS, generator=g) * 0.1
    tgts[..., 0] += feats[..., 0].float()
    return feats, tgts


def _train(micro=1):
    torch.set_num_threads(2)  # the same CPU work split in every process, so the float sums agree
    feats, tgts = _data()
    model, hist = W.train_surrogate(feats, tgts, epochs=2, batch=2, lr=1e-3, val_frac=0.0, log=None, device="cpu",
                                    conv=S.torch_conv3d, micro=micro)
    return {k: v.detach().clone() for k, v in model.params.items()}, [h["mse"] for h in hist]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        params, hist = _train()
        # by value: tensors sent through the queue would live in this process's shared memory
        q.put((rank, {k: v.numpy() for k, v in params.items()}, hist))
    finally:
        dist.destroy_process_group()


def test_two_ranks_match_one_process():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict()
    for _ in range(2):
        rank, params, hist = q.get(timeout=300)
        res[rank] = (params, hist)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    threads = torch.get_num_threads()
    try:
        single, hist1 = _train(micro=2)  # one process, the same two slices per step, gradients accumulated
    finally:
        torch.set_num_threads(threads)
    p0, h0 = res[0]
    p1, h1 = res[1]
    p0 = {k: torch.from_numpy(v) for k, v in p0.items()}
    p1 = {k: torch.from_numpy(v) for k, v in p1.items()}
    for k in single:
        assert torch.equal(p0[k], p1[k]), k  # identical updates on every rank
        assert torch.equal(p0[k], single[k]), k  # = one process accumulating the same slices
    assert h0 == h1 == hist1


def _gather_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 3 if rank == 0 else 1  # uneven shards (designs dropped by the divergence guard)
        f = torch.full((n, 2, 2, 2, S.IN_FEATURES), float(rank + 1)).to(S.BF16)
        t = torch.arange(n, dtype=torch.float32).reshape(n, 1, 1, 1, 1).expand(n, 2, 2, 2, S.OUT_FIELDS) + 10 * rank
        gf, gt = W.gather_designs(f, t.contiguous())
        q.put((rank, gf.float().numpy(), gt.numpy()))
    finally:
        dist.destroy_process_group()


def test_gather_designs_uneven_shards():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        rank, f, t = q.get(timeout=300)
        got[rank] = (f, t)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        f, t = got[rank]
        assert f.shape[0] == 4 and t.shape[0] == 4
        assert (f[:3] == 1).all() and (f[3] == 2).all()
        assert [float(t[i, 0, 0, 0, 0]) for i in range(4)] == [0.0, 1.0, 2.0, 10.0]
