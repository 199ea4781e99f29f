"""Multi-process CPU tests of the data-parallel exchange (world size 2, gloo): view assignment and
the per-step reduction of batched gradients and densification statistics."""
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from omnigs_b200 import sharding


def test_assign_views_balances_pixels_and_covers_every_view():
    sizes = [(512, 256), (1024, 512), (2048, 1024), (3072, 1536)] * 4
    for world in (1, 2, 3, 4, 8):
        a = sharding.assign_views(sizes, world)
        assert sorted(v for r in a for v in r) == list(range(len(sizes)))
        loads = [sum(sizes[v][0] * sizes[v][1] for v in r) for r in a]
        biggest = max(w * h for w, h in sizes)
        assert max(loads) - min(loads) <= biggest
        assert a == sharding.assign_views(sizes, world)  # deterministic on every rank
    assert sharding.assign_views([(64, 32)], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        sharding.assign_views(sizes, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, P, M, steps, out_q):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        red = sharding.GradientReducer(P, M, "cpu", stats=True)
        g = red.grads
        gen = torch.Generator().manual_seed(100 + rank)
        history = []
        for step in range(steps):
            # this step's gradients (written fresh) and statistics (accumulated in place)
            for t in (g.dL_dmeans3D, g.dL_dsh, g.dL_dopacity, g.dL_dscales, g.dL_drotations):
                t.copy_(torch.randn(t.shape, generator=gen))
            inc_norm = torch.rand(P, 1, generator=gen)
            inc_cnt = (torch.rand(P, 1, generator=gen) > 0.5).float()
            g.grad_accum.add_(inc_norm)
            g.denom.add_(inc_cnt)
            g.max_radii.copy_(torch.maximum(g.max_radii, torch.randint(0, 50, (P,), generator=gen).float()))
            local = {k: getattr(g, k).clone() for k in ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dscales",
                                                         "dL_drotations", "max_radii")}
            local["inc_norm"], local["inc_cnt"] = inc_norm, inc_cnt
            red.reduce()
            history.append((local, {k: getattr(g, k).clone() for k in ("dL_dmeans3D", "dL_dsh", "dL_dopacity",
                                                                        "dL_dscales", "dL_drotations",
                                                                        "grad_accum", "denom", "max_radii")}))
        # plain numpy arrays: tensors would travel as shared-memory handles that die with this process
        out_q.put((rank, [({k: v.numpy() for k, v in a.items()}, {k: v.numpy() for k, v in b.items()})
                          for a, b in history]))
    finally:
        dist.destroy_process_group()


def test_gradient_reducer_world_size_2():
    P, M, steps, world = 257, 16, 3, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, P, M, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = {r: [({k: torch.from_numpy(v) for k, v in a.items()}, {k: torch.from_numpy(v) for k, v in b.items()})
                   for a, b in h] for r, h in (q.get(timeout=120) for _ in range(world))}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    acc_norm = torch.zeros(P, 1)
    acc_cnt = torch.zeros(P, 1)
    acc_max = torch.zeros(P)
    for step in range(steps):
        loc = [results[r][step][0] for r in range(world)]
        red = [results[r][step][1] for r in range(world)]
        for k in ("dL_dmeans3D", "dL_dsh", "dL_dopacity", "dL_dscales", "dL_drotations"):
            expect = sum(l[k] for l in loc)
            for r in range(world):
                torch.testing.assert_close(red[r][k], expect, rtol=1e-6, atol=1e-6)
        acc_norm += sum(l["inc_norm"] for l in loc)
        acc_cnt += sum(l["inc_cnt"] for l in loc)
        acc_max = torch.maximum(acc_max, torch.maximum(*[l["max_radii"] for l in loc]))
        for r in range(world):
            torch.testing.assert_close(red[r]["grad_accum"], acc_norm, rtol=1e-5, atol=1e-5)
            torch.testing.assert_close(red[r]["denom"], acc_cnt, rtol=0, atol=0)
            torch.testing.assert_close(red[r]["max_radii"], acc_max, rtol=0, atol=0)
