"""Block sharding on the host (CPU only): the block ranges, the halo plan, and
a sharded run of the C oracle over gloo ranks.

The ranges follow the reference's MPI distribution
(MPI/src/BlockCommunicator.cpp:29-38).  The plan (e3d_case_shard_plan, the
same host code the shard solvers use) must pair every rank's send entries
for a peer with that peer's receive entries, entry for entry, and cover
every connexion that crosses ranks once.  Then each gloo rank runs the
oracle on its own blocks, moves the halo entries the plan lists with
all_to_all_single after every iteration, and must end with the reference's
state bit for bit (the fixtures hold the compiled reference's run).
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp
from conftest import REPO, Golden, same

from euler3d_b200 import _lib as L
from euler3d_b200 import shard
from euler3d_b200.api import Case

MULTI = ["t3_o2_gg_venk_ausm_b3", "t3_o1_ausm_b3", "t4_o2_ls_venk_roe_b2"]


def _reference_ranges(n_blocks, n_ranks):
    # BlockCommunicator::BlockCommunicator: block_process_id_[i*n + min(i, rem) + j] = i
    n, rem = n_blocks // n_ranks, n_blocks % n_ranks
    owner = [None] * n_blocks
    for i in range(n_ranks):
        for j in range(n + (i < rem)):
            owner[i * n + min(i, rem) + j] = i
    return owner


@pytest.mark.parametrize("n_blocks", [1, 2, 3, 7, 16, 160])
def test_block_ranges_follow_the_reference(n_blocks):
    for n_ranks in range(1, min(n_blocks, 9) + 1):
        fb = shard.first_blocks(n_blocks, n_ranks)
        owner = np.searchsorted(fb, np.arange(n_blocks), side="right") - 1
        assert list(owner) == _reference_ranges(n_blocks, n_ranks), (n_blocks, n_ranks)


def test_bad_ranges_are_refused(tmp_path):
    with pytest.raises(L.E3DError):
        shard.first_blocks(2, 3)  # a rank without blocks
    with pytest.raises(L.E3DError):
        shard.first_blocks(4, 0)
    case = Case(Golden("t3_o1_ausm_b3").write_case(str(tmp_path)))
    for fb in ([0, 2, 2, 3], [1, 2, 3], [0, 2, 4], [0, 3, 2]):
        with pytest.raises(L.E3DError):
            shard.plan(case, len(fb) - 1, 0, fb)
    with pytest.raises(L.E3DError):
        shard.plan(case, 2, 2)


def _connexions(case_dir, deck, n_real):
    from oracle_c import connexions_from_topology

    top = os.path.join(case_dir, os.path.basename(deck).rsplit(".", 1)[0] + ".top")
    return top, connexions_from_topology(top, n_real)


@pytest.mark.parametrize("name", MULTI)
def test_plan_pairs_send_and_receive_entries(name, tmp_path):
    g = Golden(name)
    deck = g.write_case(str(tmp_path))
    case = Case(deck)
    nb = case.n_blocks
    _, conns = _connexions(str(tmp_path), deck, [case.block_info(b).n_real for b in range(nb)])
    ghost_origin = {}
    for dest, origin, dcells, ocells in conns:
        for d, o in zip(dcells, ocells):
            ghost_origin[(dest, int(d))] = (origin, int(o))
    for n_ranks in range(1, nb + 1):
        plans = [shard.plan(case, n_ranks, r) for r in range(n_ranks)]
        fb = plans[0]["first_block"]
        owner = np.searchsorted(fb, np.arange(nb), side="right") - 1
        crossing = sum(len(d) for dest, origin, d, _ in conns if owner[dest] != owner[origin])
        assert sum(int(p["send_counts"].sum()) for p in plans) == crossing
        assert sum(int(p["recv_counts"].sum()) for p in plans) == crossing
        for a, pa in enumerate(plans):
            assert pa["send_counts"][a] == 0 and pa["recv_counts"][a] == 0
            soff = np.concatenate([[0], np.cumsum(pa["send_counts"])])
            for b, pb in enumerate(plans):
                roff = np.concatenate([[0], np.cumsum(pb["recv_counts"])])
                assert pa["send_counts"][b] == pb["recv_counts"][a]
                sent = pa["send_cells"][soff[b]:soff[b + 1]]
                got = pb["recv_cells"][roff[a]:roff[a + 1]]
                for (ob, oc), (db, dc) in zip(sent, got):
                    assert owner[ob] == a and owner[db] == b
                    assert dc >= case.block_info(int(db)).n_real  # a ghost cell of the destination block
                    assert ghost_origin[(int(db), int(dc))] == (int(ob), int(oc))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_rank(rank, world, port, name, case_dir, out):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(REPO, "tests"))
    from oracle_c import OracleBlock, OracleCase, params_from_deck

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    g = Golden(name)
    deck = [f for f in os.listdir(case_dir) if f.endswith(".deck")][0]
    case = Case(os.path.join(case_dir, deck))
    nb = case.n_blocks
    _, conns = _connexions(case_dir, deck, [case.block_info(b).n_real for b in range(nb)])
    p = shard.plan(case, world, rank)
    b0, b1 = int(p["first_block"][rank]), int(p["first_block"][rank + 1])
    local = [(d - b0, o - b0, dc, oc) for d, o, dc, oc in conns if b0 <= d < b1 and b0 <= o < b1]
    oc = OracleCase([OracleBlock.from_case(case, b) for b in range(b0, b1)], params_from_deck(case.deck), local)
    n_all = [blk.n_all for blk in oc.blocks]
    ss = [int(x) * 5 for x in p["send_counts"]]
    rs = [int(x) * 5 for x in p["recv_counts"]]

    def exchange():
        send = np.zeros((len(p["send_cells"]), 5))
        for i, (b, c) in enumerate(p["send_cells"]):
            send[i] = oc.blocks[b - b0].prim.reshape(5, n_all[b - b0])[:, c]
        recv = torch.zeros(sum(rs), dtype=torch.float64)
        dist.all_to_all_single(recv, torch.from_numpy(send.reshape(-1)), rs, ss)
        r = recv.numpy().reshape(-1, 5)
        for i, (b, c) in enumerate(p["recv_cells"]):
            oc.blocks[b - b0].prim.reshape(5, n_all[b - b0])[:, c] = r[i]

    exchange()  # the halo before the first iteration (Solver.cpp:48)
    n = len(g.hist("iter"))
    for _ in range(n):
        oc.iterate(1)
        exchange()
    out[rank] = {b0 + i: same(blk.prim, g[f"iter{n}.b{b0 + i}.prim"]) for i, blk in enumerate(oc.blocks)}
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("t3_o2_gg_venk_ausm_b3", 2), ("t3_o2_gg_venk_ausm_b3", 3),
                                        ("t4_o2_ls_venk_roe_b2", 2)])
def test_sharded_oracle_reaches_the_reference_state(name, world, tmp_path):
    Golden(name).write_case(str(tmp_path))
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_oracle_rank, args=(world, port, name, str(tmp_path), out), nprocs=world,
                           start_method="spawn", join=True)
        res = dict(out)
    blocks = {}
    for r in range(world):
        blocks.update(res[r])
    assert sorted(blocks) == list(range(Golden(name).n_blocks))
    assert all(blocks.values()), blocks
