"""Block sharding on the GPU: shard solvers over block ranges, their halo
packed and unpacked by the library's kernels, against the reference and
against the single solver.

* ``LocalShards`` runs every rank's solver in one process (device copies
  between the buffers): FP64 results are the reference's bit for bit (state,
  Cl/Cd/Cm), and the history is the single solver's exactly (the per-block
  sums are combined in block order as one GPU combines them); the FP32
  variant equals the unsharded FP32 variant bit for bit.
* ``Sharded`` over gloo with the host transport, two processes on the one GPU
  (their kernels never wait on each other; the host exchanges the buffers):
  the same results through torch.distributed.
* The library refuses an iteration before the halo has crossed, several
  iterations in one call, and e3d_solve on a shard.
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp
from conftest import REPO, Golden, max_rel, same

from euler3d_b200 import _lib as L
from euler3d_b200 import api, shard

pytestmark = pytest.mark.gpu

CASES = [("t3_o2_gg_venk_ausm_b3", 2), ("t3_o2_gg_venk_ausm_b3", 3), ("t3_o1_ausm_b3", 3),
         ("t4_o2_ls_venk_roe_b2", 2), ("t4_o2_gg_venk_roe_b2", 2)]


def _check_reference(g, h, get):
    n = len(g.hist("iter"))
    assert len(h["iter"]) == n
    for col in ("cl", "cd", "cmx", "cmy", "cmz"):
        assert same(h[col], g.hist(col)), col
    assert max_rel(h["rms"][:, 0], g.hist("rms_ro")) < 1e-12
    for b in range(g.n_blocks):
        assert same(get(b, "prim"), g[f"iter{n}.b{b}.prim"]), b


@pytest.mark.parametrize("name,ranks", CASES)
def test_local_shards_fp64_match_reference_and_single_solver(name, ranks, tmp_path):
    g = Golden(name)
    case = api.Case(g.write_case(str(tmp_path)))
    n = len(g.hist("iter"))
    run = shard.LocalShards(case, ranks)
    run.iterate(n)
    h = run.history()
    _check_reference(g, h, run.get)
    one = api.Solver(case)
    one.iterate(n)
    h1 = one.history()
    for k in ("rms", "conv", "cl", "cd"):
        assert same(h[k], h1[k]), k
    run.close()


def test_local_shards_fp32_equal_single_fp32_solver(tmp_path):
    g = Golden("t3_o2_gg_venk_ausm_b3")
    case = api.Case(g.write_case(str(tmp_path)))
    run = shard.LocalShards(case, 3, precision="fp32")
    one = api.Solver(case, precision="fp32")
    for chunk in (1, 4, 15):
        run.iterate(chunk)
        one.iterate(chunk)
    for k in ("rms", "conv", "cl", "cd", "cmx"):
        assert same(run.history()[k], one.history()[k]), k
    for b in range(3):
        assert same(run.get(b, "prim"), one.get(b, "prim")), b


def test_local_shards_full_size_16_blocks(tmp_path):
    """The 3.07M-tet, 16-block second-order case over 4 ranks of 4 blocks:
    the reference's Cl/Cd/Cm bit for bit over its 3 iterations."""
    g = Golden("bump80b16_o2_ls_venk_roe_3")
    case = api.Case(g.write_case(str(tmp_path)))
    run = shard.LocalShards(case, 4)
    run.iterate(3)
    h = run.history()
    for col in ("cl", "cd", "cmx", "cmy", "cmz"):
        assert same(h[col], g.hist(col)), col
    for q, col in enumerate(("rms_ro", "rms_uu", "rms_vv", "rms_ww", "rms_pp")):
        assert max_rel(h["rms"][:, q], g.hist(col)) < 1e-12, col
    run.close()


def test_shard_refuses_to_run_ahead_of_its_halo(tmp_path):
    case = api.Case(Golden("t4_o2_ls_venk_roe_b2").write_case(str(tmp_path)))
    s = shard.ShardSolver(case, 2, 0)
    with pytest.raises(L.E3DError) as e:
        s.iterate(1)  # the halo before the first iteration has not crossed
    assert e.value.code == -7
    assert s.send_counts[1] > 0 and s.recv_counts[1] > 0
    import torch

    n = max(int(s.send_counts.sum()), int(s.recv_counts.sum()))
    buf = torch.ones(n * 5, dtype=torch.float64, device="cuda")
    s.pack(buf.data_ptr())
    s.unpack(buf.data_ptr())  # any valid state: the refusal is about the order of calls
    with pytest.raises(L.E3DError) as e:
        s.iterate(2)
    assert e.value.code == -1
    s.iterate(1)
    with pytest.raises(L.E3DError) as e:
        s.iterate(1)
    assert e.value.code == -7
    with pytest.raises(L.E3DError):
        L.check(L.lib().e3d_solve(s._h, 10, -8.0, 1, None))
    assert s.take_flow_data().shape == (1, 1, 10)
    assert s.take_flow_data().shape == (0, 1, 10)
    s.close()


def _free_port():
    so = socket.socket()
    so.bind(("127.0.0.1", 0))
    p = so.getsockname()[1]
    so.close()
    return p


def _sharded_rank(rank, world, port, case_dir, n, out):
    import torch.distributed as dist

    sys.path.insert(0, REPO)
    from euler3d_b200 import api as A
    from euler3d_b200 import shard as S

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    deck = [f for f in os.listdir(case_dir) if f.endswith(".deck")][0]
    case = A.Case(os.path.join(case_dir, deck))
    run = S.Sharded(case, precision="fp64", transport="host", device=0)
    run.iterate(n)
    h = run.history()
    fb = run.solver.first_block
    out[rank] = {"hist": {k: np.asarray(v) for k, v in h.items()},
                 "prim": {b: run.get(b, "prim") for b in range(int(fb[rank]), int(fb[rank + 1]))}}
    run.close()
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_over_gloo_two_processes(tmp_path):
    name = "t3_o2_gg_venk_ausm_b3"
    g = Golden(name)
    g.write_case(str(tmp_path))
    n = len(g.hist("iter"))
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_sharded_rank, args=(2, port, str(tmp_path), n, out), nprocs=2, start_method="spawn",
                           join=True)
        res = dict(out)
    prim = {}
    for r in range(2):
        prim.update(res[r]["prim"])
        for k in ("rms", "cl", "cd"):
            assert same(res[r]["hist"][k], res[0]["hist"][k]), (r, k)
    _check_reference(g, res[0]["hist"], lambda b, name: prim[b])
