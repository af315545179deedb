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


class _TagSlab:
    """A slab of the step schedule with planes on the CPU: every plane holds
    a tag of (field, global plane, version), so a plane that arrives from a
    neighbour shows where it came from.  The phases check what the reference
    exchanges before them and write new tags after them."""

    N = 4  # doubles per plane

    def __init__(self, rank, ranks, nzs):
        import torch
        self.rank, self.ranks, self.nz = rank, ranks, nzs[rank]
        self.kst = sum(nzs[:rank])
        self.planes = {}
        for f in range(3):
            for k in range(-1, self.nz + 3):
                self.planes[(f, k)] = torch.full((self.N,), -1.0, dtype=torch.float64)
        for k in range(self.nz + 1):
            self.planes[(3, k)] = torch.full((self.N,), -1.0, dtype=torch.float64)
        for f in range(4, 10):
            self.planes[(f, 0)] = torch.zeros(self.N if f < 8 else 1, dtype=torch.float64)
        self.version = 0
        self.failures = []

    @staticmethod
    def tag(field, kg, version):
        return 1e6 * field + 10.0 * kg + version

    def tensor(self, field, k=0):
        return self.planes[(field, k)]

    def _expect(self, field, k, value, what):
        got = float(self.planes[(field, k)][0])
        if got != value:
            self.failures.append(f"rank {self.rank} {what}: plane ({field},{k}) = {got}, expected {value}")

    def _write_interior(self, fields):
        for f in fields:
            for k in range(1, self.nz + 1):
                self.planes[(f, k)].fill_(self.tag(f, self.kst + k, self.version))

    def check_velocity_halos(self, version):
        lo = -1 if self.rank > 0 else 1
        hi = self.nz + 2 if self.rank < self.ranks - 1 else self.nz
        for f in range(3):
            for k in range(lo, hi + 1):
                self._expect(f, k, self.tag(f, self.kst + k, version), "velocity halo")

    def rk(self):
        self.version += 1
        self._write_interior(range(3))
        self.planes[(8, 0)].fill_(self.rank + 1.0)

    def mean_finish(self):
        total = self.ranks * (self.ranks + 1) / 2
        self._expect(8, 0, total, "Mean_h sum")

    def rhs_sweep(self):
        if self.rank > 0:  # w plane nz of the lower neighbour, for the divergence at k = 1
            self._expect(2, 0, self.tag(2, self.kst, self.version), "w halo")
        self.planes[(4, 0)].fill_(self.tag(4, self.kst, self.version))

    def pdd_iface(self):
        if self.rank < self.ranks - 1:
            self._expect(5, 0, self.tag(4, self.kst + self.nz, self.version), "tvar")
        self.planes[(6, 0)].fill_(self.tag(6, self.rank, self.version))

    def finish(self):
        if self.rank > 0:
            self._expect(7, 0, self.tag(6, self.rank - 1, self.version), "y1")
        self.planes[(3, 0)].fill_(self.tag(3, self.kst, self.version))

    def correct(self):
        if self.rank < self.ranks - 1:
            self._expect(3, self.nz, self.tag(3, self.kst + self.nz, self.version), "p halo")


def _schedule_rank(rank, world, port, nz, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    from powerllel_channel_b200 import slab as S
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    nzs = S.slab_sizes(nz, world)[1]
    me = _TagSlab(rank, world, nzs)
    tr = S.DistTransport(me, tensor_of=me.tensor)
    marks = []
    for _ in range(2):
        S.step([me], tr, nzs, marks.append)
        me.check_velocity_halos(me.version)
    q.put((rank, me.failures, marks))
    dist.destroy_process_group()


@pytest.mark.parametrize("world,nz", [(2, 8), (3, 10)])
def test_slab_step_schedule_moves_every_plane(world, nz):
    """the whole step's exchanges over gloo: the Mean_h sum, the w halo, the
    PDD planes, the pressure halo and two velocity planes each way reach the
    phase that reads them, on every rank, in the same order of marks"""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_schedule_rank, args=(r, world, port, nz, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    failures = [f for _, fs, _ in res for f in fs]
    assert not failures, failures[:10]
    marks = {r: m for r, _, m in res}
    assert all(m == marks[0] for m in marks.values())
    assert marks[0][:4] == ["rk_fused", "x_mean", "mean_finish", "x_w"]
    assert marks[0][-1] == "x_vel" and len(marks[0]) == 2 * 12
