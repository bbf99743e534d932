"""z-slab decomposition of the step over several GPUs (one process each).

The grid is cut into slabs of whole z planes, one per rank.  A rank steps the
planes it owns plus a halo of HALO planes on each side that touches another
rank, as a grid of its own: the step's kernels see that grid's first and last
planes as walls, and the values they compute there are wrong, but the error
travels at most 14 planes inward in one step with ten Jacobi sweeps
(predictor 1, ten Jacobi sweeps 10 -- their right-hand side reaches one plane
up --, correction 1 down, z sweep of the volume fraction 3: the reach of each
phase of voftrial1.cu:1361-1401 along z; halo_for).  After every step
each rank sends the planes it owns next to a neighbour to that neighbour,
which writes them over its halo: one point-to-point exchange of five fields
(F, u, v, w, p) per step, and the owned planes of every rank hold exactly the
values the single-GPU step would (bit for bit: the same kernels, the same
operands).  The halo planes cost redundant work; the exchange is one message
per neighbour and field (NCCL over NVLink between GPUs, gloo on CPU).

A rank owns at least HALO planes, so a halo comes from one neighbour only.
Reductions (the liquid volume) sum over owned planes and are all-reduced.
Only VOF_MODE_PLAIN: the convergent modes' pressure solve couples the whole
grid in every iteration.

The step itself is not the reference's concern (voftrial1.cu runs one GPU);
this is the multi-GPU layer over the C-ABI (vof_get_planes / vof_put_planes
/ vof_reduce_range / vof_run).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

HALO = 16
STATE = ("F", "u", "v", "w", "p")


@dataclass(frozen=True)
class Slab:
    """Global interior planes (1-based, inclusive) of one rank."""
    own0: int   # first owned plane
    own1: int   # last owned plane
    lo: int     # first plane of the rank's grid (own0 - halo below, or 1)
    hi: int     # last plane of the rank's grid (own1 + halo above, or nz)

    @property
    def nz(self) -> int:
        return self.hi - self.lo + 1

    def local(self, k: int) -> int:
        """Local plane index of global plane k (ghost planes included)."""
        return k - self.lo + 1


def halo_for(jacobi_iters: int) -> int:
    """Planes a step invalidates next to a cut, with two to spare: the
    predictor 1, the Jacobi sweeps one each (their right-hand side adds one
    above), the correction 1 below, the z sweep 3 -- jacobi_iters + 4 on each
    side."""
    return max(HALO, jacobi_iters + 6)


def plan(nz: int, nranks: int, halo: int = HALO) -> list[Slab]:
    """Owned planes as even as possible; halo planes where a neighbour is."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    base, extra = divmod(nz, nranks)
    out = []
    k = 1
    for r in range(nranks):
        n = base + (1 if r < extra else 0)
        if nranks > 1 and n < halo:
            raise ValueError(f"{nz} planes over {nranks} ranks: slabs of {n} planes, fewer than the halo ({halo})")
        own0, own1 = k, k + n - 1
        lo = own0 - halo if r > 0 else 1
        hi = own1 + halo if r < nranks - 1 else nz
        out.append(Slab(own0, own1, lo, hi))
        k += n
    return out


def local_params(prm, slab: Slab):
    """The rank's grid: the global parameters with nz (and kmax, nTot) of the
    slab.  dz and dzi stay the global values (no re-derivation from Lz)."""
    q = prm.copy()
    q.nz = slab.nz
    q.kmax = q.kmin + q.nz - 1
    q.nTot = (q.nx + 2) * (q.ny + 2) * (q.nz + 2)
    q.Lz = float(np.float32(prm.dz) * np.float32(slab.nz))
    return q


def local_state(state: dict, slab: Slab) -> dict:
    """Global fields (nz+2, ny+2, nx+2) -> the slab's (ghost planes lo-1, hi+1)."""
    return {k: np.ascontiguousarray(state[k][slab.lo - 1:slab.hi + 2]) for k in STATE}


class Exchange:
    """The planes one rank sends and receives after each step."""

    def __init__(self, slabs: list[Slab], rank: int):
        self.rank = rank
        s = slabs[rank]
        self.sends, self.recvs = [], []  # (peer, local k0, nk)
        if rank > 0:
            below = slabs[rank - 1]
            n_up = below.hi - below.own1  # planes of mine the rank below holds as halo
            self.sends.append((rank - 1, s.local(s.own0), n_up))
            self.recvs.append((rank - 1, s.local(s.lo), s.own0 - s.lo))
        if rank < len(slabs) - 1:
            above = slabs[rank + 1]
            n_dn = above.own0 - above.lo
            self.sends.append((rank + 1, s.local(s.own1 - n_dn + 1), n_dn))
            self.recvs.append((rank + 1, s.local(s.own1 + 1), s.hi - s.own1))


class TorchComm:
    """Point-to-point exchange and sums through torch.distributed (NCCL for
    CUDA tensors between GPUs, gloo for CPU tensors)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def exchange(self, sends, recvs):
        """sends/recvs: lists of (peer, tensor); every send is matched by the
        peer's recv of the same shape."""
        dist = self.dist
        ops = [dist.P2POp(dist.isend, t, self._global(p), group=self.group) for p, t in sends]
        ops += [dist.P2POp(dist.irecv, t, self._global(p), group=self.group) for p, t in recvs]
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def sum(self, x: float, device=None) -> float:
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=device)
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())

    def _global(self, p):
        return p if self.group is None else self.dist.get_global_rank(self.group, p)


class SlabRank:
    """One rank of the decomposition over an engine with the Solver interface
    (vof_b200.Solver on a GPU; the tests also drive a CPU engine).

    engine_factory(local_params) -> engine with upload_state, step(istep),
    run(istep0, n), get_planes(field, k0, nk, device_ptr=...),
    put_planes(field, k0, device_ptr=..., nk=...), reduce_range(what, k0, k1),
    state(); plane buffers are torch tensors on `device`."""

    def __init__(self, prm, comm, engine_factory, device="cpu", halo: int | None = None):
        import torch

        if prm.mode != 0 or prm.surface_tension != 0:
            raise ValueError("the slab decomposition runs the plain step only")
        self.torch = torch
        self.prm = prm
        self.comm = comm
        self.slabs = plan(prm.nz, comm.size, halo if halo is not None else halo_for(prm.jacobi_iters))
        self.slab = self.slabs[comm.rank]
        self.lprm = local_params(prm, self.slab)
        self.engine = engine_factory(self.lprm)
        self.device = device
        self.ex = Exchange(self.slabs, comm.rank)
        plane = (prm.ny + 2) * (prm.nx + 2)
        self.sbuf = {(p, k0): torch.empty((len(STATE), nk * plane), dtype=torch.float32, device=device)
                     for p, k0, nk in self.ex.sends}
        self.rbuf = {(p, k0): torch.empty((len(STATE), nk * plane), dtype=torch.float32, device=device)
                     for p, k0, nk in self.ex.recvs}

    # -- state ----------------------------------------------------------------
    def upload_global(self, state: dict):
        self.engine.upload_state(**local_state(state, self.slab))

    def owned(self) -> dict:
        """The planes this rank holds the values of: its owned interior planes,
        plus the global ghost plane beside the first (last) slab.  Reference
        layout; concatenated over the ranks they are the global fields."""
        st = self.engine.state()
        a, b = self.slab.local(self.slab.own0), self.slab.local(self.slab.own1)
        if self.comm.rank == 0:
            a -= 1
        if self.comm.rank == self.comm.size - 1:
            b += 1
        return {k: st[k][a:b + 1] for k in STATE}

    # -- halo exchange --------------------------------------------------------
    def _nk(self, buf) -> int:
        return buf.shape[1] // ((self.prm.ny + 2) * (self.prm.nx + 2))

    def pack(self):
        """Copy the owned planes the neighbours hold as halo into the send buffers."""
        dev = self.device != "cpu"
        for (p, k0), buf in self.sbuf.items():
            nk = self._nk(buf)
            for q, f in enumerate(STATE):
                if dev:
                    self.engine.get_planes(f, k0, nk, device_ptr=buf[q].data_ptr())
                else:
                    buf[q].copy_(self.torch.from_numpy(np.ascontiguousarray(self.engine.get_planes(f, k0, nk))
                                                       .reshape(-1)))

    def unpack(self):
        """Write the received planes over the halo."""
        dev = self.device != "cpu"
        for (p, k0), buf in self.rbuf.items():
            nk = self._nk(buf)
            for q, f in enumerate(STATE):
                if dev:
                    self.engine.put_planes(f, k0, device_ptr=buf[q].data_ptr(), nk=nk)
                else:
                    self.engine.put_planes(f, k0, buf[q].numpy().reshape(nk, self.prm.ny + 2, self.prm.nx + 2))

    def exchange(self):
        self.pack()
        self.comm.exchange([(p, b) for (p, _), b in self.sbuf.items()], [(p, b) for (p, _), b in self.rbuf.items()])
        self.unpack()

    # -- stepping -------------------------------------------------------------
    def step(self, istep: int):
        self.engine.step(istep)
        self.exchange()

    def run(self, istep0: int, nsteps: int):
        for s in range(nsteps):
            self.engine.run(istep0 + s, 1)
            self.exchange()

    def volume(self) -> float:
        a, b = self.slab.local(self.slab.own0), self.slab.local(self.slab.own1)
        v = self.engine.reduce_range("volume", a, b)
        return self.comm.sum(v, device=self.device if self.device != "cpu" else None)


class LocalComm:
    """Rank and size of one member of a LocalGroup (no messages of its own)."""

    def __init__(self, rank: int, size: int):
        self.rank, self.size = rank, size


class LocalGroup:
    """All ranks of a decomposition in one process -- several contexts on one
    GPU, or CPU engines: the same slabs, halos and plane copies as ranks on
    separate GPUs, with the messages as copies between the ranks' buffers."""

    def __init__(self, prm, nranks: int, engine_factory, device="cpu", halo: int | None = None):
        self.ranks = [SlabRank(prm, LocalComm(r, nranks), engine_factory, device, halo) for r in range(nranks)]

    def upload_global(self, state: dict):
        for r in self.ranks:
            r.upload_global(state)

    def exchange(self):
        for r in self.ranks:
            r.pack()
        for r in self.ranks:
            for (p, _), buf in r.sbuf.items():
                peer = self.ranks[p]
                dst = next(b for (q, _), b in peer.rbuf.items() if q == r.comm.rank)
                dst.copy_(buf)
        for r in self.ranks:
            r.unpack()

    def run(self, istep0: int, nsteps: int):
        for s in range(nsteps):
            for r in self.ranks:
                r.engine.run(istep0 + s, 1)
            self.exchange()

    def state(self) -> dict:
        parts = [r.owned() for r in self.ranks]
        return {k: np.concatenate([p[k] for p in parts]) for k in STATE}

    def volume(self) -> float:
        tot = 0.0
        for r in self.ranks:
            a, b = r.slab.local(r.slab.own0), r.slab.local(r.slab.own1)
            tot += r.engine.reduce_range("volume", a, b)
        return tot
