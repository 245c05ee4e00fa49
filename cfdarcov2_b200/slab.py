"""x-slab decomposition of one structured mesh over the ranks of a process group.

The legacy multi-process design of the reference distributes mesh nodes
over MPI ranks, exchanges the neighbour values each operator needs with
MPI_Isend / MPI_Irecv (legacy/cfdarcho_main.cpp:158-207) and takes the
global time step with MPI_Allreduce(MIN) (legacy/fvm.cpp:785).  Here the
split follows the mesh's slowest axis: rank r owns the x planes
[x0, x1) of a balanced split, and holds one ghost plane on each side that has
a neighbour rank.  A step is

  1. exchange: for every field, the first and last owned planes go to the
     neighbour ranks and their planes come back into the ghost planes
     (point-to-point isend / irecv; NCCL over NVLink on GPUs, gloo on CPUs);
  2. the ordinary single-mesh step on the local array (ghost planes
     included): a 7-point stencil's owned cells see exactly the neighbour
     values of the undivided mesh, so they get the same bits; the ghost
     planes' own updates are discarded by the next exchange.

Scalar reductions cross ranks through all_reduce: the minimum of the ranks'
dt (the reference's CFL step), and sums of FP64 totals.  Remote planes
always land in this rank's own memory before a kernel reads them: no kernel
reads another GPU's memory.

The step itself is the caller's (a function (a, b) -> None that advances the
local array a into b), so the same driver runs the library's kernels on GPUs
and any other implementation of the step."""
from __future__ import annotations


def split(nx: int, world: int, rank: int) -> tuple[int, int]:
    """Balanced x range [x0, x1) of `rank`: plane counts differ by at most one."""
    if not 0 <= rank < world or nx < world:
        raise ValueError(f"cannot split {nx} planes over {world} ranks (rank {rank})")
    return rank * nx // world, (rank + 1) * nx // world


class Slab:
    """One rank's part of an nx x ny x nz mesh carrying `nfields` fields
    stored field after field (the library's state layout)."""

    def __init__(self, nx: int, ny: int, nz: int, nfields: int, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nx, self.ny, self.nz, self.nf = int(nx), int(ny), int(nz), int(nfields)
        self.x0, self.x1 = split(self.nx, self.world, self.rank)
        self.glo = 1 if self.rank > 0 else 0               # ghost plane below x0
        self.ghi = 1 if self.rank < self.world - 1 else 0  # ghost plane at x1
        self.lnx = self.x1 - self.x0 + self.glo + self.ghi  # local planes
        self.plane = self.ny * self.nz
        self.lx0 = self.x0 - self.glo  # global index of local plane 0

    @property
    def local_elems(self) -> int:
        return self.nf * self.lnx * self.plane

    def _peer(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def _plane(self, local, f, i):
        """Local plane i of field f (a contiguous view)."""
        o = (f * self.lnx + i) * self.plane
        return local[o: o + self.plane]

    def scatter(self, full, out):
        """This rank's planes (ghosts included) of the undivided state `full`
        into the local array `out`."""
        n3 = self.nx * self.plane
        for f in range(self.nf):
            src = full[f * n3 + self.lx0 * self.plane: f * n3 + (self.lx0 + self.lnx) * self.plane]
            out[f * self.lnx * self.plane: (f + 1) * self.lnx * self.plane].copy_(src)
        return out

    def exchange(self, local):
        """Fills the ghost planes of `local` from the neighbour ranks."""
        ops = []
        d = self.dist
        for f in range(self.nf):
            if self.glo:
                ops.append(d.P2POp(d.isend, self._plane(local, f, 1), self._peer(self.rank - 1), self.group))
                ops.append(d.P2POp(d.irecv, self._plane(local, f, 0), self._peer(self.rank - 1), self.group))
            if self.ghi:
                ops.append(d.P2POp(d.isend, self._plane(local, f, self.lnx - 2), self._peer(self.rank + 1), self.group))
                ops.append(d.P2POp(d.irecv, self._plane(local, f, self.lnx - 1), self._peer(self.rank + 1), self.group))
        if ops:
            for w in d.batch_isend_irecv(ops):
                w.wait()

    def owned(self, local):
        """The owned planes of every field, as one tensor per field."""
        return [local[(f * self.lnx + self.glo) * self.plane: (f * self.lnx + self.lnx - self.ghi) * self.plane]
                for f in range(self.nf)]

    def gather(self, local, full=None):
        """Assembles the undivided state on rank 0 (into `full`, which rank 0
        passes); the other ranks send their owned planes and return None."""
        import torch
        d = self.dist
        mine = torch.cat(self.owned(local))
        if self.rank != 0:
            d.send(mine.contiguous(), self._peer(0), self.group)
            return None
        n3 = self.nx * self.plane
        for r in range(self.world):
            a, b = split(self.nx, self.world, r)
            if r == 0:
                buf = mine
            else:
                buf = torch.empty(self.nf * (b - a) * self.plane, dtype=local.dtype, device=local.device)
                d.recv(buf, self._peer(r), self.group)
            k = (b - a) * self.plane
            for f in range(self.nf):
                full[f * n3 + a * self.plane: f * n3 + b * self.plane].copy_(buf[f * k: (f + 1) * k])
        return full

    def run(self, a, b, steps: int, step):
        """`steps` steps a -> b -> a ..., each after a ghost exchange; returns
        the array holding the final state."""
        for _ in range(int(steps)):
            self.exchange(a)
            step(a, b)
            a, b = b, a
        return a

    def min_dt(self, dt: float, device=None) -> float:
        """The smallest dt over the ranks (MPI_Allreduce(MIN) of the reference)."""
        import torch
        t = torch.tensor([float(dt)], dtype=torch.float64, device=device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
        return float(t.item())

    def sum_fp64(self, values, device=None):
        """Element-wise FP64 sums over the ranks (totals of conserved fields)."""
        import torch
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return [float(v) for v in t.tolist()]

    def local_vertices(self, vertices):
        """The vertex rows of this rank's local planes (ghosts included) from
        the undivided (nx+1)(ny+1)(nz+1) x 3 vertex array, x slowest."""
        vp = (self.ny + 1) * (self.nz + 1)
        return vertices[self.lx0 * vp: (self.lx0 + self.lnx + 1) * vp]
