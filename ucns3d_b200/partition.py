"""Partitions of a prepared mesh, one engine per rank, halo transfers per RK stage.

UCNS3D splits the mesh with METIS (src/main.f90:103-137, the partition read
in src/io.f90) and, inside every RK stage, exchanges the halo's cell means
(EXCHANGE_HIGHER, src/communications.f90:1085-1246) and the quadrature-point
values of the partition faces (EXHBOUNDHIGHER, :1745-1956) over MPI before
the fluxes.  Here:

* `rcb` splits the cells by recursive coordinate bisection of their centres
  (METIS is not available; any partition vector can be passed instead).
* `PartitionPlan` gives each rank its local cells: the owned cells, their
  face neighbours (ring 1), every stencil member of both and the face
  neighbours of ring 1.  Every cell whose face values an owned residual uses
  is then reconstructed locally from exact data, so only cell states cross
  between ranks, once per stage, and no face-value exchange is needed.
  Local cells are numbered in increasing global index, so each face keeps its
  owning side and the face fluxes are the whole mesh's bit for bit.
* `PartitionMesh` is a rank's mesh: the whole mesh's geometry and tables
  sliced to the local cells, neighbour and stencil indices renumbered.  At a
  cut (a local cell whose neighbour is not local) the face becomes a
  symmetry face and stencil members that are not local point at the cell
  itself; both only touch cells outside owned + ring 1, whose results no
  owned residual reads and whose states the next transfer overwrites.
* `HaloEngine` steps one rank: per stage, the send rows are packed on the
  device (`ucg_halo_pack`), moved to the peers (`torch.distributed` point to
  point over NCCL, or gloo for host tensors), unpacked (`ucg_halo_unpack`),
  and the stage runs (`ucg_rk3_stage`); the CFL time step is the minimum of
  the ranks' local minima (CALCULATE_CFL is per cell).
* `LocalCluster` runs several ranks' engines in one process on one device,
  the transfers being device copies between their buffers, each stage's
  packs finished before its unpacks (no kernel waits for another).
"""
from __future__ import annotations

import numpy as np

from . import _native as N

MF = 6  # faces per cell (UCG_MAX_FACES)


def rcb(centres: np.ndarray, nparts: int) -> np.ndarray:
    """Recursive coordinate bisection: part index per cell, parts of equal
    size within one cell.  Each split cuts the longest extent of its cells'
    centres at the count quantile of the two halves' shares (nparts need not
    be a power of two); ties are broken by the cell index, so the result is
    deterministic."""
    n = len(centres)
    if nparts < 1:
        raise ValueError("nparts must be at least 1")
    part = np.zeros(n, dtype=np.int32)

    def split(idx, first, k):
        if k == 1 or len(idx) == 0:
            part[idx] = first
            return
        x = centres[idx]
        axis = int(np.argmax(x.max(0) - x.min(0)))
        order = idx[np.lexsort((idx, x[:, axis]))]
        k1 = k // 2
        m = (len(idx) * k1) // k
        split(order[:m], first, k1)
        split(order[m:], first + k1, k - k1)

    split(np.arange(n, dtype=np.int64), 0, nparts)
    return part


def _mark(n: int, idx: np.ndarray) -> np.ndarray:
    """The distinct non-negative entries of idx, increasing (a mark array
    instead of a sort: stencil arrays reach 10^8 entries)."""
    m = np.zeros(n, dtype=bool)
    m[idx[idx >= 0]] = True
    return np.flatnonzero(m)


def _neighbours(neigh: np.ndarray, nfaces: np.ndarray, cells: np.ndarray) -> np.ndarray:
    nb = neigh[cells]
    valid = np.arange(MF)[None, :] < nfaces[cells][:, None]
    return _mark(len(neigh), np.where(valid, nb, -1))


class PartitionPlan:
    """The local cells and transfer lists of every rank of partition `part`
    of a prepared mesh.  Every rank builds the same plan from the same
    inputs.  For rank r: `cells[r]` (global indices, increasing),
    `owned[r]` (mask over them), `core[r]` (mask: owned and ring 1), and for
    each peer q `recv[r][q]` / `send[r][q]`: local indices of the halo cells
    that q owns, and of the owned cells that q receives, both in increasing
    global index, so that send[q][r] and recv[r][q] name the same cells in
    the same order."""

    def __init__(self, mesh, part: np.ndarray):
        part = np.asarray(part, dtype=np.int32)
        n = mesh.ncells
        if part.shape != (n,) or part.min() < 0:
            raise ValueError("part must give a non-negative part index per cell")
        self.base, self.part = mesh, part
        self.nparts = int(part.max()) + 1
        if np.bincount(part, minlength=self.nparts).min() == 0:
            raise ValueError("every part from 0 to max(part) must own at least one cell")
        g, r = mesh.geometry(), mesh.recon()
        neigh, nfaces, sten = g["neigh"], g["nfaces"], r["stencil"]
        self.cells, self.owned, self.core = [], [], []
        for k in range(self.nparts):
            owned = np.flatnonzero(part == k)
            ring1 = np.setdiff1d(_neighbours(neigh, nfaces, owned), owned)
            core = np.union1d(owned, ring1)
            local = np.union1d(np.union1d(core, _mark(n, sten[core])), _neighbours(neigh, nfaces, ring1))
            self.cells.append(local)
            self.owned.append(part[local] == k)
            self.core.append(np.isin(local, core))
        self.recv = [dict() for _ in range(self.nparts)]
        self.send = [dict() for _ in range(self.nparts)]
        for k in range(self.nparts):
            loc = self.cells[k]
            halo = np.flatnonzero(~self.owned[k])
            owners = part[loc[halo]]
            for q in np.unique(owners):
                q = int(q)
                rows = halo[owners == q]  # increasing global index, as loc is
                self.recv[k][q] = rows.astype(np.int32)
                # the same cells in q's numbering
                self.send[q][k] = np.searchsorted(self.cells[q], loc[rows]).astype(np.int32)
        for k in range(self.nparts):
            for q, rows in self.send[k].items():
                assert np.array_equal(self.cells[k][rows], self.cells[q][self.recv[q][k]])
                assert self.owned[k][rows].all()

    def peers(self, rank: int) -> list:
        """Ranks that rank `rank` exchanges with, increasing."""
        return sorted(set(self.recv[rank]) | set(self.send[rank]))

    def roles(self, rank: int) -> np.ndarray:
        """Per local cell of rank `rank`: 0 owned, 1 ring 1, 2 the rest of the
        halo (ucg_set_cell_roles)."""
        r = np.full(len(self.cells[rank]), 2, dtype=np.int8)
        r[self.core[rank]] = 1
        r[self.owned[rank]] = 0
        return r

    def local(self, rank: int, a: np.ndarray) -> np.ndarray:
        """Rows of a whole-mesh per-cell array that rank `rank` holds."""
        return np.ascontiguousarray(a[self.cells[rank]])

    def assemble(self, owned_rows: list) -> np.ndarray:
        """The whole-mesh array from each rank's owned rows (rank order)."""
        first = owned_rows[0]
        out = np.empty((self.base.ncells,) + first.shape[1:], dtype=first.dtype)
        for k, rows in enumerate(owned_rows):
            out[self.cells[k][self.owned[k]]] = rows
        return out


class PartitionMesh:
    """Rank `rank`'s mesh of a `PartitionPlan`: the interface the engine and
    the oracle take from a prepared mesh (see the module notes for the cut
    faces and stencils)."""

    def __init__(self, plan: PartitionPlan, rank: int):
        base = plan.base
        cells = plan.cells[rank]
        n = base.ncells
        self.base, self.cells, self.rank = base, cells, rank
        self.prepared = True
        self.sizes = base.sizes
        self.scheme, self.iorder, self.ees = base.scheme, base.iorder, base.ees
        loc = np.full(n, -1, dtype=np.int64)
        loc[cells] = np.arange(len(cells))
        g = base.geometry()
        self._g = {k: (np.ascontiguousarray(v[cells]) if isinstance(v, np.ndarray) else v) for k, v in g.items()}
        nb = self._g["neigh"]
        nf = self._g["nfaces"]
        live = np.arange(MF)[None, :] < nf[:, None]
        mapped = np.where(nb >= 0, loc[np.maximum(nb, 0)], -1)
        cut = live & (nb >= 0) & (mapped < 0)
        core = plan.core[rank]
        if cut[core].any():
            raise AssertionError("a cell of owned + ring 1 lost a face neighbour")
        self._g["neigh"] = mapped.astype(np.int32)
        bc = self._g["bc"].copy()
        bc[cut] = 3  # symmetry: a valid ghost for a face whose flux nothing reads
        self._g["bc"] = bc
        self.cut_faces = int(cut.sum())
        r = base.recon()
        self._r = dict(r)
        st = r["stencil"][cells]
        ms = np.where(st >= 0, loc[np.maximum(st, 0)], -1)
        lost = (st >= 0) & (ms < 0)
        if lost[core].any():
            raise AssertionError("a stencil of owned + ring 1 is not local")
        own_idx = np.broadcast_to(np.arange(len(cells))[:, None, None], ms.shape)
        ms = np.where(lost, own_idx, ms)
        self._r["stencil"] = np.ascontiguousarray(ms.astype(np.int32))
        if r["table_id"] is not None:
            self._r["table_id"] = np.ascontiguousarray(r["table_id"][cells])
        else:  # per-cell matrix sets move with their cells
            for k in ("invmat", "invmat2", "indicator", "indicator2"):
                if r.get(k) is not None:
                    self._r[k] = np.ascontiguousarray(r[k][cells])

    @property
    def ncells(self) -> int:
        return len(self.cells)

    @property
    def ntables(self) -> int:
        return self._r["ntables"]

    def fill_config(self, cfg: N.UcgConfig) -> N.UcgConfig:
        return self.base.fill_config(cfg)

    def geometry_struct(self) -> N.UcgGeometry:
        import ctypes as C
        g, s = self._g, N.UcgGeometry()
        s.ncells = self.ncells
        for k in ("nfaces", "face_type", "neigh", "neigh_face", "bc", "qperm", "admis", "full"):
            setattr(s, k, N.ptr(g[k], C.c_int32))
        for k in ("face_angle", "face_area", "dih", "qpoints", "volume", "minedge", "invccjac", "basis_mean"):
            if g[k] is not None:
                setattr(s, k, N.ptr(g[k], C.c_double))
        return s

    def recon_struct(self) -> N.UcgRecon:
        import ctypes as C
        r, s = self._r, N.UcgRecon()
        s.first, s.count = 0, self.ncells
        s.stencil = N.ptr(r["stencil"], C.c_int32)
        s.ntables = r["ntables"]
        if r["table_id"] is not None:
            s.table_id = N.ptr(r["table_id"], C.c_int32)
        for k in ("invmat", "invmat2", "indicator", "indicator2"):
            if r.get(k) is not None:
                setattr(s, k, N.ptr(r[k], C.c_double))
        return s

    def geometry(self) -> dict:
        return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self._g.items()}

    def recon(self) -> dict:
        return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self._r.items()}

    def centres(self) -> np.ndarray:
        return self.base.centres()[self.cells]


class HaloLists:
    """One rank's transfer layout: its peers, the send rows (owned cells,
    peer after peer) and receive rows (halo cells, peer after peer) as local
    indices, and each peer's slice of them."""

    def __init__(self, plan: PartitionPlan, rank: int):
        self.peers = plan.peers(rank)
        empty = np.zeros(0, np.int32)
        send = [plan.send[rank].get(q, empty) for q in self.peers]
        recv = [plan.recv[rank].get(q, empty) for q in self.peers]
        self.send = np.concatenate(send).astype(np.int32) if send else empty
        self.recv = np.concatenate(recv).astype(np.int32) if recv else empty
        self._so = np.concatenate([[0], np.cumsum([len(x) for x in send])]).astype(np.int64)
        self._ro = np.concatenate([[0], np.cumsum([len(x) for x in recv])]).astype(np.int64)

    def send_slice(self, q: int) -> slice:
        i = self.peers.index(q)
        return slice(int(self._so[i]), int(self._so[i + 1]))

    def recv_slice(self, q: int) -> slice:
        i = self.peers.index(q)
        return slice(int(self._ro[i]), int(self._ro[i + 1]))


def transfer(lists: HaloLists, sendbuf, recvbuf, group=None):
    """Each peer's slice of `sendbuf` to it and its slice of `recvbuf` from
    it (torch tensors [rows][5] on the process group's device), point to
    point.  Returns once the receives are complete (on CUDA: once the current
    stream waits for them)."""
    import torch.distributed as dist
    ops = []
    for q in lists.peers:
        a, b = sendbuf[lists.send_slice(q)], recvbuf[lists.recv_slice(q)]
        if len(a):
            ops.append(dist.P2POp(dist.isend, a, q, group=group))
        if len(b):
            ops.append(dist.P2POp(dist.irecv, b, q, group=group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class HaloEngine:
    """One rank's engine on its partition.  `comm` is the `torch.distributed`
    process group of the transfers (None: the default group).  `restrict`
    (default) gives the engine the cells' roles, so that it reconstructs
    owned + ring 1 only and steps the owned cells; without it the whole
    local mesh is reconstructed and stepped (the same owned results)."""

    def __init__(self, plan: PartitionPlan, rank: int, cfg, device: int = 0, comm=None, restrict: bool = True):
        import torch
        from .engine import Engine
        self.plan, self.rank, self.device = plan, rank, device
        self.mesh = PartitionMesh(plan, rank)
        self.engine = Engine(self.mesh, cfg, device=device, roles=plan.roles(rank) if restrict else None)
        self.lists = HaloLists(plan, rank)
        self.peers = self.lists.peers
        if plan.nparts > 1 and not self.peers:
            # the grouped point-to-point call of every stage (NCCL) must
            # include every rank, so a rank without halo rows would hang it
            self.engine.close()
            raise ValueError(f"rank {rank} shares no halo with another part (a disconnected piece of the mesh)")
        self.engine.halo_set(self.lists.send, self.lists.recv)
        dev = torch.device("cuda", device)
        self.sendbuf = torch.empty((len(self.lists.send), 5), dtype=torch.float64, device=dev)
        self.recvbuf = torch.empty((len(self.lists.recv), 5), dtype=torch.float64, device=dev)
        self.stream = torch.cuda.ExternalStream(self.engine.stream_ptr, device=dev)
        self.comm = comm
        self.restrict = restrict

    def close(self):
        self.engine.close()

    # ------------------------------------------------------------ state
    def set_state(self, U: np.ndarray):
        """The whole mesh's state [n][5]; the rank keeps its local rows."""
        self.engine.set_state(self.plan.local(self.rank, U))

    def owned_state(self) -> np.ndarray:
        return self.engine.get_state()[self.plan.owned[self.rank]]

    # -------------------------------------------------------- transfers
    def send_rows(self, q: int):
        return self.sendbuf[self.lists.send_slice(q)]

    def recv_rows(self, q: int):
        return self.recvbuf[self.lists.recv_slice(q)]

    def pack(self, stage: int):
        if len(self.sendbuf):
            self.engine.halo_pack(stage, self.sendbuf.data_ptr())

    def unpack(self, stage: int):
        if len(self.recvbuf):
            self.engine.halo_unpack(stage, self.recvbuf.data_ptr())

    def exchange(self, stage: int):
        """The halo rows of stage `stage`'s input state from their owners
        (one rank per process, `torch.distributed` point to point)."""
        import torch
        self.pack(stage)
        with torch.cuda.stream(self.stream):  # ordered after the pack, before the unpack
            transfer(self.lists, self.sendbuf, self.recvbuf, self.comm)
        self.unpack(stage)

    # ---------------------------------------------------------- stepping
    def rk3_step(self, dt: float):
        """One RUNGE_KUTTA3 step of size dt on this rank (every rank calls it)."""
        for s in (1, 2, 3):
            self.exchange(s)
            self.engine.rk3_stage(s, dt)

    def compute_dt(self, cfl: float) -> float:
        """CALCULATE_CFL of the whole mesh: the halo of U^n brought up to date,
        this rank's minimum, then the minimum over the ranks."""
        import torch
        import torch.distributed as dist
        self.exchange(1)
        dt = self.engine.calculate_cfl(cfl)
        if not dist.is_initialized():  # one process holds the whole mesh
            return dt
        t = torch.tensor([dt], dtype=torch.float64, device=self.sendbuf.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.comm)
        return float(t.item())


    def wall_loads(self, centre=None) -> np.ndarray:
        """COMPUTEFORCE of the whole mesh: the halo of U^n brought up to date,
        this rank's walls (those of its owned cells: the engine has the
        roles), then the sum over the ranks.  `centre` is the whole mesh's
        cell centres (n, 3) for the moments, or None."""
        import torch
        import torch.distributed as dist
        if not self.restrict:
            raise ValueError("the wall loads of a rank need the cell roles (restrict=True)")
        self.exchange(1)
        loads = self.engine.wall_loads(None if centre is None else self.plan.local(self.rank, centre))
        if not dist.is_initialized():
            return loads
        t = torch.tensor(loads, dtype=torch.float64, device=self.sendbuf.device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.comm)
        return t.cpu().numpy()


class LocalCluster:
    """All ranks of a plan as engines in this process on one device: each
    stage packs every rank, copies the rows between the ranks' buffers, then
    unpacks and runs the stage on every rank.  Every kernel is ordered by the
    host, so none waits for another rank's."""

    def __init__(self, plan: PartitionPlan, cfg, device: int = 0, restrict: bool = True):
        self.plan = plan
        self.ranks = [HaloEngine(plan, k, cfg, device=device, restrict=restrict) for k in range(plan.nparts)]

    def close(self):
        for h in self.ranks:
            h.close()

    def set_state(self, U: np.ndarray):
        for h in self.ranks:
            h.set_state(U)

    def get_state(self) -> np.ndarray:
        return self.plan.assemble([h.owned_state() for h in self.ranks])

    def exchange(self, stage: int):
        import torch
        for h in self.ranks:
            h.pack(stage)
        torch.cuda.synchronize()
        for h in self.ranks:
            for q in h.peers:
                dst = h.recv_rows(q)
                if len(dst):
                    dst.copy_(self.ranks[q].send_rows(h.rank))
        torch.cuda.synchronize()
        for h in self.ranks:
            h.unpack(stage)

    def rk3_step(self, dt: float):
        for s in (1, 2, 3):
            self.exchange(s)
            for h in self.ranks:
                h.engine.rk3_stage(s, dt)

    def compute_dt(self, cfl: float) -> float:
        self.exchange(1)
        return min(h.engine.calculate_cfl(cfl) for h in self.ranks)

    def wall_loads(self, centre=None) -> np.ndarray:
        """The ranks' wall loads added in rank order (the engines need the
        roles: restrict=True)."""
        if not all(h.restrict for h in self.ranks):
            raise ValueError("the wall loads of a rank need the cell roles (restrict=True)")
        self.exchange(1)
        return sum(h.engine.wall_loads(None if centre is None else self.plan.local(h.rank, centre))
                   for h in self.ranks)
