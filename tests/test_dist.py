"""Replicas across ranks (CPU, gloo, world size 2): each rank serves its own
partition of the requests on its own engine (here the host-emulation build)
with no exchange on the data path; only the finished results' metrics are
gathered on rank 0."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from profess_b200 import build, native, serving, workloads as wl
    eng = native.Engine(build.EMU_PATH)
    rids = serving.partition(list(range(5)), rank, world)
    srv = serving.Server(eng, hbm_budget=10 ** 12, ticks_per_poll=4)
    for i in rids:
        c = wl.fcc_al((1, 1, 1), sigma_ang=0.05, grid=(16, 16, 16), seed=i)
        srv.submit(serving.Request(rid=i, cell=c, arrival=0.0, mode=serving.MODE_FP64, seed=i))
    res = srv.run_until_done(timeout=600)
    mine = {r.rid: float(r.energy[0]) for r in res}
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        allres = {}
        for g in gathered:
            allres.update(g)
        out.put(allres)
    dist.barrier()
    dist.destroy_process_group()
    eng.close()


def test_two_rank_replicas():
    from profess_b200 import build
    build.build_emu()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    allres = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(allres) == [0, 1, 2, 3, 4]
    assert len(set(round(v, 9) for v in allres.values())) == 5  # distinct displaced cells
