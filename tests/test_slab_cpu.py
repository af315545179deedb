"""The multi-GPU z-slab schedule on CPU: two and four gloo ranks.

powerllel_channel_b200.slab.pdd_solve is the PDD part of the slab step: each
rank sweeps its partition, sends its first swept plane down, solves the
interface with its upper neighbour, sends y3 up and corrects.  Here every
rank's compute is the oracle's partition of the restated PDD solve (a CPU
stand-in with the slab's phase names and planes) and the planes move over
torch.distributed with the gloo backend, so the test checks the partitioning
(decomp_2d.c:261-283) and the exchange schedule (psolve_trid's two
MPI_Sendrecv calls, mod_poisson_solver.c:415-417, 444-446) against the
reference's own multi-rank PDD build: the golden fixtures were made by the
reference with p_col forked ranks.  Bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, name, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    os.environ.setdefault("OMP_NUM_THREADS", "2")
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    from oracle import oracle as O
    from powerllel_channel_b200 import slab as S
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    nx, ny, nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    ppe = O.PPE(nx, ny, nz, float(d["dx"]), float(d["dy"]), d["dzf"], nparts=world)
    st, sz = S.slab_sizes(nz, world)
    me = O.SlabPPE(ppe, rank, d["rhs"][st[rank]:st[rank] + sz[rank]])
    assert (me.kst, me.nz) == (st[rank], sz[rank])
    tr = S.DistTransport(me, tensor_of=me.tensor)
    S.pdd_solve([me], tr, sz)
    parts = [None] * world
    dist.all_gather_object(parts, me.out)
    if rank == 0:
        q.put(np.concatenate(parts, axis=0))
    dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("ppe_pdd2_32x24x32", 2), ("ppe_pdd4_32x24x30", 4)])
def test_slab_pdd_schedule_matches_reference_ranks(name, world):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert np.array_equal(got, d["p"])


def test_slab_sizes_follow_decomp_2d():
    from powerllel_channel_b200 import slab as S
    assert S.slab_sizes(30, 4) == ([0, 7, 14, 22], [7, 7, 8, 8])
    assert S.slab_sizes(32, 2) == ([0, 16], [16, 16])
    assert S.slab_sizes(512, 8) == ([64 * r for r in range(8)], [64] * 8)
