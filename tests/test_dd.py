"""Domain decomposition over a grid of ranks, without a GPU: the plan
(qcuDDPlan) against qcu's rank grid, the pairing of every rank's face
exchange (qcuDDSchedule), and that exchange carried out by two gloo ranks,
checked against the neighbours on the global lattice."""
import itertools
import os

import numpy as np
import pytest

from ddref import coord_of

GRIDS = [[2, 1, 1, 1], [1, 2, 1, 1], [1, 1, 2, 1], [1, 1, 1, 2], [2, 2, 1, 1], [1, 3, 2, 1], [2, 2, 2, 2],
         [4, 1, 1, 3]]
LOC = [4, 6, 2, 4]


@pytest.fixture(scope="module")
def q():
    import qcu_b200

    return qcu_b200


@pytest.mark.parametrize("grid", GRIDS)
def test_plan_is_qcus_rank_grid(q, grid):
    n = int(np.prod(grid))
    faces = [LOC[1] * LOC[2] * LOC[3] // 2, LOC[0] // 2 * LOC[2] * LOC[3], LOC[0] // 2 * LOC[1] * LOC[3],
             LOC[0] // 2 * LOC[1] * LOC[2]]
    for r in range(n):
        p = q.dd_plan(LOC, grid, r)
        c = coord_of(r, grid)
        assert p["nranks"] == n and p["rank"] == r and p["coord"] == c
        for d in range(4):
            cf, cb = list(c), list(c)
            cf[d] = (c[d] + 1) % grid[d]
            cb[d] = (c[d] - 1) % grid[d]
            assert coord_of(p["fwd"][d], grid) == cf and coord_of(p["bwd"][d], grid) == cb
            assert q.dd_plan(LOC, grid, p["fwd"][d])["bwd"][d] == r
            assert p["face"][d] == (faces[d] if grid[d] > 1 else 0)


def test_plan_rejects_bad_grids(q):
    with pytest.raises(q.QcuError, match="even"):
        q.dd_plan([4, 3, 4, 4], [1, 2, 1, 1], 0)
    with pytest.raises(q.QcuError, match="rank"):
        q.dd_plan(LOC, [2, 1, 1, 1], 2)


@pytest.mark.parametrize("grid", GRIDS)
def test_schedules_pair_up(q, grid):
    """Every send meets, in order, a receive of the same size on the peer; a
    low face (slot 0) lands in the backward rank's slot 0 (its forward
    halo), a high face in the forward rank's slot 1."""
    n = int(np.prod(grid))
    sched = {r: q.dd_schedule(LOC, grid, r) for r in range(n)}
    plan = {r: q.dd_plan(LOC, grid, r) for r in range(n)}
    taken = {(r, k): False for r in range(n) for k in range(len(sched[r]))}
    for r in range(n):
        for kind, d, slot, peer, cnt in sched[r]:
            if kind != "send":
                continue
            match = next(k for k, op in enumerate(sched[peer])
                         if op[0] == "recv" and op[3] == r and not taken[(peer, k)])
            taken[(peer, match)] = True
            _, d2, slot2, _, cnt2 = sched[peer][match]
            assert (d2, slot2, cnt2) == (d, slot, cnt)
            assert peer == (plan[r]["bwd"][d] if slot == 0 else plan[r]["fwd"][d])
            assert cnt == 6 * plan[r]["face"][d]
    assert all(taken[(r, k)] for r in range(n) for k, op in enumerate(sched[r]) if op[0] == "recv")


def _face_index(d, x, y, z, t, loc):
    Lxh, Ly, Lz = loc[0] // 2, loc[1], loc[2]
    if d == 0:
        return ((t * Lz + z) * Ly + y) >> 1
    if d == 1:
        return (t * Lz + z) * Lxh + (x >> 1)
    if d == 2:
        return (t * Ly + y) * Lxh + (x >> 1)
    return (z * Ly + y) * Lxh + (x >> 1)


def _gloo_worker(rank, world, port, grid, out_q):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import qcu_b200 as q

        plan = q.dd_plan(LOC, grid, rank)
        sched = q.dd_schedule(LOC, grid, rank)
        c = plan["coord"]
        G = [LOC[d] * grid[d] for d in range(4)]

        def gid(x, y, z, t):  # global lexicographic id of a global coordinate
            return ((t % G[3] * G[2] + z % G[2]) * G[1] + y % G[1]) * G[0] + x % G[0]

        sites = list(itertools.product(range(LOC[0]), range(LOC[1]), range(LOC[2]), range(LOC[3])))
        errors = 0
        for parity in (0, 1):
            q_in = 1 - parity
            send = {(d, s): torch.full((max(plan["face"][d], 1), 12), -1.0, dtype=torch.float64)
                    for d in range(4) for s in (0, 1)}
            halo = {(d, s): torch.full((max(plan["face"][d], 1), 12), -2.0, dtype=torch.float64)
                    for d in range(4) for s in (0, 1)}
            for x, y, z, t in sites:
                if (x + y + z + t) & 1 != q_in:
                    continue
                g = gid(c[0] * LOC[0] + x, c[1] * LOC[1] + y, c[2] * LOC[2] + z, c[3] * LOC[3] + t)
                pos = (x, y, z, t)
                for d in range(4):
                    if grid[d] == 1:
                        continue
                    f = _face_index(d, x, y, z, t, LOC)
                    if pos[d] == 0:
                        send[(d, 0)][f] = g
                    if pos[d] == LOC[d] - 1:
                        send[(d, 1)][f] = g
            ops = []
            for kind, d, s, peer, cnt in sched:
                buf = send[(d, s)] if kind == "send" else halo[(d, s)]
                assert cnt == buf.numel() // 2
                ops.append(dist.P2POp(dist.isend if kind == "send" else dist.irecv, buf, peer))
            for w in dist.batch_isend_irecv(ops):
                w.wait()
            for x, y, z, t in sites:
                if (x + y + z + t) & 1 != parity:
                    continue
                X, Y, Z, T = c[0] * LOC[0] + x, c[1] * LOC[1] + y, c[2] * LOC[2] + z, c[3] * LOC[3] + t
                pos = (x, y, z, t)
                for d in range(4):
                    if grid[d] == 1:
                        continue
                    f = _face_index(d, x, y, z, t, LOC)
                    step = [int(k == d) for k in range(4)]
                    if pos[d] == LOC[d] - 1:  # forward hop: the forward neighbour's site
                        want = gid(X + step[0], Y + step[1], Z + step[2], T + step[3])
                        errors += int(not torch.all(halo[(d, 0)][f] == want))
                    if pos[d] == 0:  # backward hop
                        want = gid(X - step[0], Y - step[1], Z - step[2], T - step[3])
                        errors += int(not torch.all(halo[(d, 1)][f] == want))
        out_q.put((rank, errors))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("grid", [[2, 1, 1, 1], [1, 2, 1, 1], [1, 1, 2, 1], [1, 1, 1, 2]])
def test_gloo_two_ranks_exchange_faces(grid):
    """Two processes carry out their schedules with gloo point-to-point; every
    received face site is the global neighbour the hop needs."""
    import multiprocessing as mp
    import socket

    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out_q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, grid, out_q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(out_q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: 0, 1: 0}
