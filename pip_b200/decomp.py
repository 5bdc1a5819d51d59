"""Spatial domain decomposition of the two-fluid step over ranks (the MPI layer of PIP,
MPI_rot.f90, rebuilt for one process per GPU).

The reference splits the grid into blocks (``set_mpi_pos``, MPI_rot.f90:43-88; the 1D split
``flag_mpi_split = 1`` puts every rank along x), gives each rank its own block with ghost
cells (``set_mpi``, :11-41), its own coordinates (``set_coordinate``'s MPI branch,
Model_rot.f90:410-417), its neighbours (``set_mpi_neighbor``, :90-126), fills the ghost
layers between blocks after every RK stage (``mpi_bnd`` inside ``PIPbnd``,
Boundary_rot.f90:34-52; two ``MPI_Sendrecv`` per direction, :128-339) and reduces dt (MIN)
and cmax (MAX) over ranks in ``cfl`` (Scheme_rot.f90:200-210).

Here a 2D grid is split along y (rows stay whole, so a y message is a run of contiguous
rows) and a 1D grid along x.  Each rank's block is a ``Context`` told its neighbours
(``pip_set_neighbors``).  A step is either driven from the host (``run``):

    cfl on every block -> MIN over ranks -> dt;  cmax = MAX over ranks of safety*min(d)/dt
    stage 1 -> halo exchange -> stage 2 -> halo exchange -> cfl (the rewrite of main.f90:47)

or queued on the device (``run_device``, pip_dev_*): stage 1 takes dt and cmax from the cfl
candidates, stage 2 computes the next step's candidates, and the MIN/MAX over ranks is an
allreduce of those device words between the steps, so nothing waits on the host.

The exchange has the reference's two phases per direction: every block sends its upper
interior layers to the neighbour above and receives its lower ghost layers from the
neighbour below, then the reverse.  Messages are packed and unpacked on the device
(``pip_halo_pack`` / ``pip_halo_unpack``) and moved by ``torch.distributed`` point-to-point
(NCCL over NVLink between GPUs), or, for several blocks held by one process, by a device
copy.

Blocks are engines with the methods ``cfl() -> (dt, cmax)``, ``stage(k, dt, cmax)``,
``halo_bytes(face)``, ``message_bytes(face)``, ``buffer(nbytes)``,
``pack(face, buf) -> nbytes``, ``unpack(face, buf, nbytes)``, ``stream()`` (a context
manager ordering the transfers with the block's own work), ``has_nan() -> bool``,
``download()`` and ``close()``; ``DeviceBlock`` is the one on a GPU context.  A device
block's stages, packing and unpacking are queued on its context's stream and the NCCL
transfers are issued on that stream, so a step waits on the host only in its two cfl
calls.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .params import Settings

FACE_NAMES = ("x-", "x+", "y-", "y+")


# ---------------------------------------------------------------------- the split
def split_axis(s: Settings) -> int:
    """0 (x) for 1D grids, 1 (y) for 2D grids."""
    return 0 if s.ndim == 1 else 1


@dataclasses.dataclass
class Block:
    """One rank's part of the grid."""
    rank: int
    world: int
    settings: Settings            # the rank's own grid (interior cells of the block)
    neighbor: Tuple[int, int, int, int]
    lo: int                       # first global interior index along the split axis
    n: int                        # interior cells along the split axis

    @property
    def sg(self) -> float:
        """safety*min(dx, dy, dz) of the block (the numerator of cfl's cmax)."""
        _, _, _, dx, dy, dz = self.settings.coordinates()
        return self.settings.safety * min(dx.min(), dy.min(), dz.min())


def block_of(s: Settings, world: int, rank: int) -> Block:
    """set_mpi / set_mpi_pos / set_mpi_neighbor / set_coordinate for rank ``rank`` of
    ``world`` blocks along the split axis."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of %d" % (rank, world))
    ax = split_axis(s)
    total = s.ix0 if ax == 0 else s.jx0
    if total % world:
        raise ValueError("%d cells along %s do not divide into %d blocks"
                         % (total, "xy"[ax], world))
    n = total // world
    # set_coordinate's MPI branch (Model_rot.f90:410-417)
    start, end = list(s.start), list(s.end)
    length = end[ax] - start[ax]
    ds = 1.0 / world
    start[ax] = start[ax] + ds * rank * length
    end[ax] = start[ax] + ds * length
    kw = {"ix0": n} if ax == 0 else {"jx0": n}
    local = s.overrides(start=tuple(start), end=tuple(end), **kw)
    # set_mpi_neighbor (MPI_rot.f90:90-126): periodic faces wrap around the ranks
    nb = [-1, -1, -1, -1]
    if world > 1:
        lo_face, hi_face = 2 * ax, 2 * ax + 1
        nb[lo_face] = rank - 1
        nb[hi_face] = rank + 1
        if rank == 0:
            nb[lo_face] = world - 1 if s.flag_bnd[lo_face] == 1 else -1
        if rank == world - 1:
            nb[hi_face] = 0 if s.flag_bnd[hi_face] == 1 else -1
    return Block(rank, world, local, tuple(nb), rank * n, n)


def scatter(s: Settings, U: np.ndarray, world: int, rank: int) -> np.ndarray:
    """The rank's block of a global state (planes, jx, ix) with ghosts: its interior plus
    margin layers on each side along the split axis, taken from the global array (the
    neighbours' interior cells, or the global ghost cells at the ends)."""
    b = block_of(s, world, rank)
    ax = split_axis(s)
    m = s.margin[ax]
    sl = slice(b.lo, b.lo + b.n + 2 * m)
    return np.ascontiguousarray(U[:, :, sl] if ax == 0 else U[:, sl, :])


def gather(s: Settings, parts: Sequence[np.ndarray]) -> np.ndarray:
    """The global state from every rank's block (rank order): interiors side by side, the
    global ghost layers from the first and last blocks."""
    world = len(parts)
    ax = split_axis(s)
    m = s.margin[ax]
    out = []
    for r, p in enumerate(parts):
        n = (p.shape[2] if ax == 0 else p.shape[1]) - 2 * m
        a = m if r > 0 else 0
        e = m + n + (m if r == world - 1 else 0)
        out.append(p[:, :, a:e] if ax == 0 else p[:, a:e, :])
    return np.ascontiguousarray(np.concatenate(out, axis=2 if ax == 0 else 1))


# ---------------------------------------------------------------------- transports
class TorchComm:
    """Reductions and point-to-point messages between processes through
    ``torch.distributed`` (NCCL for device buffers, gloo for host buffers).  staged: the
    transport takes host buffers only (gloo) while the blocks' buffers are on the device;
    each message and reduction then goes through a host copy, ordered after the work
    queued on the current stream."""

    def __init__(self, device=None, group=None, staged: bool = False):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.torch = torch
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device = device if device is not None else "cpu"
        self.staged = staged

    def barrier(self) -> None:
        self.dist.barrier(group=self.group)

    def allreduce(self, value: float, op: str) -> float:
        t = self.torch.tensor([value], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN if op == "min" else self.dist.ReduceOp.MAX,
                             group=self.group)
        return float(t.item())

    def allreduce_sums(self, values) -> List[float]:
        """mpi_allreduce(..., MPI_SUM) of a few doubles (BiCGstabMPI's scalars)."""
        t = self.torch.tensor(list(values), dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return [float(v) for v in t.tolist()]

    def reduce_candidates(self, pairs) -> None:
        """cfl's MIN/MAX allreduces on device memory: pairs = [(t_min, t_max)] of this
        process's blocks (one), reduced in place over the ranks on the current stream."""
        for t_min, t_max in pairs:
            for t, op in ((t_min, self.dist.ReduceOp.MIN), (t_max, self.dist.ReduceOp.MAX)):
                if self.staged and t.is_cuda:
                    h = t.cpu()                      # after the stream's queued work
                    self.dist.all_reduce(h, op=op, group=self.group)
                    t.copy_(h)
                else:
                    self.dist.all_reduce(t, op=op, group=self.group)

    def exchange(self, sends, recvs) -> None:
        """sends: [(src_rank, dst_rank, tensor)], recvs: [(dst_rank, src_rank, tensor)] for
        this process's blocks; at most one message per ordered pair of ranks.  The sends and
        receives go out as one batch (one NCCL group), so two ranks that send to each other
        do not wait on each other's receive."""
        P2POp = self.dist.P2POp
        if self.staged:
            hs = [(dst, t.cpu() if t.is_cuda else t) for _, dst, t in sends]
            hr = [(src, t, self.torch.empty_like(t, device="cpu") if t.is_cuda else t)
                  for _, src, t in recvs]
            ops = [P2POp(self.dist.irecv, h, src, self.group) for src, _, h in hr]
            ops += [P2POp(self.dist.isend, h, dst, self.group) for dst, h in hs]
            for q in self.dist.batch_isend_irecv(ops):
                q.wait()
            for _, t, h in hr:
                if t is not h:
                    t.copy_(h)
            return
        ops = [P2POp(self.dist.irecv, t, src, self.group) for _, src, t in recvs]
        ops += [P2POp(self.dist.isend, t, dst, self.group) for _, dst, t in sends]
        # with NCCL the transfer starts after the current stream's work (the packing) and
        # wait() makes the current stream wait for it (no host block)
        for q in self.dist.batch_isend_irecv(ops):
            q.wait()


class LocalComm:
    """Every block in this process (several GPU contexts on one device, or host engines):
    reductions over the blocks and messages as device/host copies."""

    rank = 0

    def allreduce(self, value: float, op: str) -> float:
        return value

    def allreduce_sums(self, values) -> List[float]:
        return [float(v) for v in values]

    def barrier(self) -> None:
        pass

    def reduce_candidates(self, pairs) -> None:
        if len(pairs) < 2:     # one block: the reduction is the identity
            return
        import torch
        torch.cuda.synchronize()
        lo = torch.stack([a for a, _ in pairs]).min(dim=0).values
        hi = torch.stack([b for _, b in pairs]).max(dim=0).values
        for a, b in pairs:
            a.copy_(lo)
            b.copy_(hi)
        torch.cuda.synchronize()

    def exchange(self, sends, recvs) -> None:
        box = {(src, dst): t for src, dst, t in sends}
        sync = any(t.is_cuda for _, _, t in recvs)
        if sync:       # the blocks' streams differ: packing done before the copies ...
            import torch
            torch.cuda.synchronize()
        for dst, src, t in recvs:
            t.copy_(box[(src, dst)])
        if sync:       # ... and the copies before the unpacking
            torch.cuda.synchronize()


# ---------------------------------------------------------------------- engines
class _DeviceArray:
    """A device address as a CUDA-array-interface object (a zero-copy torch view)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i8", "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


def _device_int64(ptr: int, n: int, device):
    import torch
    return torch.as_tensor(_DeviceArray(ptr, n), device=device)


class DeviceBlock:
    """A rank's block on a GPU context (``pip_set_neighbors`` + ``pip_stage`` +
    ``pip_halo_pack/unpack``)."""

    def __init__(self, block: Block, U_h: np.ndarray, U_m: np.ndarray, device: int = 0,
                 eta: Optional[np.ndarray] = None):
        """eta: the block's part of a fixed resistivity field (flag_resi).  By default a
        localised field (resi_type 1) is made from the block's own coordinates, as each
        rank's set_resistivity does (Res_rot.f90:29-35); pass the scattered global field to
        match a single-domain run bit for bit."""
        import torch
        from .capi import Context
        self.torch = torch
        self.block = block
        self.ctx = Context(block.settings)
        self.ctx.set_neighbors(block.neighbor)
        self.ctx.upload(U_h, U_m)
        if eta is None and block.settings.flag_resi and block.settings.resi_type:
            # resi_type 2, 3 set once at the prologue (flag_resi 21, 31): from the block's
            # state, its ghost layers as uploaded
            eta = block.settings.eta_field(U_m if block.settings.resi_type >= 2 else None)
        if eta is not None:
            self.ctx.set_resistivity(eta)
        self.device = torch.device("cuda", device)
        self.mixed = block.settings.precision != 0
        self.last_stage = 0
        self._stream = torch.cuda.ExternalStream(self.ctx.stream, device=self.device)
        self._side = {}

    def cfl(self) -> Tuple[float, float]:
        return self.ctx.cfl()

    def stage(self, k: int, dt: float, cmax: float) -> None:
        self.ctx.stage(k, dt, cmax)
        self.last_stage = k

    def dev_stage(self, k: int) -> None:
        self.ctx.dev_stage(k)
        self.last_stage = k

    def dev_stage_split(self, k: int):
        """Stage k with its first and last tile rows (what the y exchange sends) on a
        high-priority stream, concurrent with the middle rows; returns an event that fires
        when the boundary rows are done."""
        bs = self.ctx.dev_stage_split(k)
        self.last_stage = k
        if bs not in self._side:
            self._side[bs] = self.torch.cuda.ExternalStream(bs, device=self.device)
        ev = self.torch.cuda.Event()
        ev.record(self._side[bs])
        return ev

    def wait(self, ev) -> None:
        """The context stream waits for ev."""
        self._stream.wait_event(ev)

    def set_halo_stream(self, stream) -> None:
        """Queue pack and unpack on `stream` (a torch stream; None: the context stream)."""
        self.ctx.set_halo_stream(stream.cuda_stream if stream is not None else 0)

    def candidates(self):
        """int64 views of the device cfl candidates: (2 to MIN, 4 to MAX)."""
        a, b = self.ctx.dev_candidates()
        return _device_int64(a, 2, self.device), _device_int64(b, 4, self.device)

    def message_bytes(self, face: int) -> int:
        """Length of the message of face f for the state the last stage wrote: the FP32-mixed
        form's stage-1 array holds one FP32 value per cell, every other state 8 bytes."""
        n = self.ctx.halo_bytes(face)
        return n // 2 if (self.mixed and self.last_stage == 1) else n

    def buffer(self, nbytes: int):
        return self.torch.empty(nbytes, dtype=self.torch.uint8, device=self.device)

    def halo_bytes(self, face: int) -> int:
        return self.ctx.halo_bytes(face)

    def pack(self, face: int, buf) -> int:
        return self.ctx.halo_pack(face, buf.data_ptr())

    def unpack(self, face: int, buf, nbytes: int) -> None:
        self.ctx.halo_unpack(face, buf.data_ptr(), nbytes)

    def stream(self):
        """Context manager that makes torch work (the NCCL transfers) run in order with the
        context's stream."""
        return self.torch.cuda.stream(self._stream)

    # conduction of the decomposed run (pip_hcd_*): vector 0 x, 1 r, 2 Ap
    def hcd_begin(self, dt: float) -> Tuple[float, float]:
        return self.ctx.hcd_begin(dt)

    def hcd_phase(self, phase: int, c0: float = 0.0, c1: float = 0.0) -> Tuple[float, float]:
        return self.ctx.hcd_phase(phase, c0, c1)

    def hcd_row_bytes(self) -> int:
        return self.ctx.hcd_row_bytes()

    def hcd_pack(self, vec: int, face: int, buf) -> int:
        self.ctx.hcd_pack(vec, face, buf.data_ptr())
        return self.ctx.hcd_row_bytes()

    def hcd_unpack(self, vec: int, face: int, buf) -> None:
        self.ctx.hcd_unpack(vec, face, buf.data_ptr())

    def hcd_end(self, iters: int) -> None:
        self.ctx.hcd_end(iters)

    def has_nan(self) -> bool:
        return bool(self.ctx.status()[1])

    def download(self) -> Tuple[np.ndarray, np.ndarray]:
        return self.ctx.download()

    def alpha_c(self) -> np.ndarray:
        return self.ctx.alpha_c()

    def close(self) -> None:
        self.ctx.close()


# ---------------------------------------------------------------------- the driver
class DecomposedRun:
    """The time loop of main.f90:31-68 over decomposed blocks.  ``engines`` are the blocks
    this process holds (one per process with ``TorchComm``, all of them with
    ``LocalComm``)."""

    def __init__(self, engines: Sequence, comm, divb: bool):
        self.engines = list(engines)
        self.comm = comm
        self.divb = divb
        self.time = 0.0
        self.steps = 0
        self.dt_history: List[float] = []
        self._send: Dict[Tuple[int, int], object] = {}
        self._recv: Dict[Tuple[int, int], object] = {}
        for e in self.engines:
            for f in range(4):
                if e.block.neighbor[f] >= 0:
                    n = e.halo_bytes(f)
                    self._send[(e.block.rank, f)] = e.buffer(n)
                    self._recv[(e.block.rank, f)] = e.buffer(n)

    def halo(self, stream=None) -> None:
        """mpi_bnd (MPI_rot.f90:128-339): per split direction, phase 1 sends the upper
        interior layers up and fills the lower ghost layers from below; phase 2 the
        reverse.  With `stream` (a torch stream) the transfers run on it (the engines' pack
        and unpack must have been pointed at it too)."""
        for d in (0, 1):
            for send_face in (2 * d + 1, 2 * d):
                recv_face = send_face ^ 1
                sends, recvs = [], []
                for e in self.engines:
                    r = e.block.rank
                    if e.block.neighbor[send_face] >= 0:
                        buf = self._send[(r, send_face)]
                        n = e.pack(send_face, buf)
                        sends.append((r, e.block.neighbor[send_face], buf[:n]))
                    if e.block.neighbor[recv_face] >= 0:
                        n = e.message_bytes(recv_face)
                        recvs.append((r, e.block.neighbor[recv_face], self._recv[(r, recv_face)][:n]))
                if not sends and not recvs:
                    continue
                if stream is not None:
                    with self.engines[0].torch.cuda.stream(stream):
                        self.comm.exchange(sends, recvs)
                elif len(self.engines) == 1:
                    with self.engines[0].stream():
                        self.comm.exchange(sends, recvs)
                else:
                    self.comm.exchange(sends, recvs)
                for e in self.engines:
                    r = e.block.rank
                    if e.block.neighbor[recv_face] >= 0:
                        e.unpack(recv_face, self._recv[(r, recv_face)], e.message_bytes(recv_face))

    def _hcd_halo(self, vec: int) -> None:
        """mpiBND(v, 1) of a BiCGstab vector: one row across each exchanged y face, in the
        two phases of halo()."""
        for send_face in (3, 2):
            recv_face = send_face ^ 1
            sends, recvs = [], []
            for e in self.engines:
                r = e.block.rank
                if e.block.neighbor[send_face] >= 0:
                    buf = self._hc_send[(r, send_face)]
                    n = e.hcd_pack(vec, send_face, buf)
                    sends.append((r, e.block.neighbor[send_face], buf[:n]))
                if e.block.neighbor[recv_face] >= 0:
                    buf = self._hc_recv[(r, recv_face)]
                    recvs.append((r, e.block.neighbor[recv_face], buf))
            if not sends and not recvs:
                continue
            if len(self.engines) == 1:
                with self.engines[0].stream():
                    self.comm.exchange(sends, recvs)
            else:
                self.comm.exchange(sends, recvs)
            for e in self.engines:
                r = e.block.rank
                if e.block.neighbor[recv_face] >= 0:
                    e.hcd_unpack(vec, recv_face, self._hc_recv[(r, recv_face)])

    def _sums(self, parts) -> List[float]:
        """SUM over this process's blocks (in block order), then over the ranks."""
        a0 = 0.0
        a1 = 0.0
        for s0, s1 in parts:
            a0 += s0
            a1 += s1
        return self.comm.allreduce_sums([a0, a1])

    def conduction(self, dt: float, hc_error: float, hc_max: int) -> Tuple[int, float]:
        """post_step's HC over dt (Solver_rot.f90:296-303) as BiCGstabMPI (HC_rot.f90:303-466)
        on the device blocks, then the state's exchange (the closing PIPbnd).  Returns
        (iterations, relative residual); every rank takes the same steps."""
        if not hasattr(self, "_hc_send"):
            self._hc_send, self._hc_recv = {}, {}
            for e in self.engines:
                for f in (2, 3):
                    if e.block.neighbor[f] >= 0:
                        n = e.hcd_row_bytes()
                        self._hc_send[(e.block.rank, f)] = e.buffer(n)
                        self._hc_recv[(e.block.rank, f)] = e.buffer(n)
        tr, tb = self._sums([e.hcd_begin(dt) for e in self.engines])
        self._hcd_halo(1)
        for e in self.engines:
            e.hcd_phase(0)
        count = 0
        while np.sqrt(tr / tb) > hc_error and count <= hc_max:
            au, ad = self._sums([e.hcd_phase(1) for e in self.engines])
            alpha = au / ad
            self._hcd_halo(2)
            ou, od = self._sums([e.hcd_phase(2, alpha) for e in self.engines])
            omega = ou / od
            for e in self.engines:
                e.hcd_phase(3, alpha, omega)
            bu, tr = self._sums([e.hcd_phase(4) for e in self.engines])
            self._hcd_halo(1)
            beta = bu / au * alpha / omega
            for e in self.engines:
                e.hcd_phase(5, beta, omega)
            count += 1
        for e in self.engines:
            e.hcd_end(count)
        self.halo()
        self.hc_iterations = count
        return count, float(np.sqrt(tr / tb))

    def step(self) -> float:
        """cfl; run_solver with PIPbnd's exchange after each stage (and post_step's
        conduction with flag_heat = 1); cfl (main.f90:36-47)."""
        dt = min(e.cfl()[0] for e in self.engines)
        dt = self.comm.allreduce(dt, "min")
        cmax = 0.0
        if self.divb:
            cmax = self.comm.allreduce(max(e.block.sg / dt for e in self.engines), "max")
        for k in (1, 2):
            for e in self.engines:
                e.stage(k, dt, cmax)
            self.halo()
        s = self.engines[0].block.settings
        if s.flag_heat == 1 and any(n >= 0 for e in self.engines for n in e.block.neighbor):
            # (a block without neighbours conducts inside its stage 2, as pip_stage does)
            self.conduction(dt, s.hc_error, s.hc_max)
        for e in self.engines:
            e.cfl()
        self.time += dt
        self.steps += 1
        self.dt_history.append(dt)
        return dt

    def _stage_overlapped(self, k: int) -> None:
        """Stage k with its y exchange overlapped: the first and last tile rows on a
        high-priority stream, then the exchange on the halo stream while the middle rows
        compute on the block streams."""
        hs = self._halo_stream
        for e in self.engines:
            hs.wait_event(e.dev_stage_split(k))
        self.halo(stream=hs)
        done = self.engines[0].torch.cuda.Event()
        done.record(hs)
        for e in self.engines:
            e.wait(done)

    def run_device(self, nsteps: int, check_every: int = 64, overlap: bool = False) -> int:
        """nsteps steps with dt, cmax and time on the device (pip_dev_*): per step stage 1,
        exchange, stage 2 (with the next step's cfl candidates), exchange, MIN/MAX of the
        candidates over ranks -- all queued on the block streams, no host wait; the host
        checks the stop flags every check_every steps.  overlap (2D y-split): each exchange
        runs on a stream of its own while the stage's middle tile rows compute.  Returns 0,
        3 (NaN) or 4 (dt floor), the same on every rank."""
        overlap = overlap and all(e.block.settings.ndim == 2 for e in self.engines)
        if overlap:
            torch = self.engines[0].torch
            self._halo_stream = torch.cuda.Stream(device=self.engines[0].device)
            for e in self.engines:
                e.set_halo_stream(self._halo_stream)
        if not getattr(self, "_scaled", False):
            sg = self.comm.allreduce(max(e.block.sg for e in self.engines), "max")
            for e in self.engines:
                e.ctx.set_cmax_scale(sg)
            self._scaled = True
        pairs = [e.candidates() for e in self.engines]

        def reduce():
            if len(self.engines) == 1:
                with self.engines[0].stream():
                    self.comm.reduce_candidates(pairs)
            else:
                self.comm.reduce_candidates(pairs)

        for e in self.engines:
            e.ctx.dev_begin(nsteps=nsteps)
        reduce()
        for n in range(nsteps):
            if overlap:
                self._stage_overlapped(1)
                self._stage_overlapped(2)
            else:
                for e in self.engines:
                    e.dev_stage(1)
                self.halo()
                for e in self.engines:
                    e.dev_stage(2)
                self.halo()
            reduce()
            if check_every and (n + 1) % check_every == 0 and n + 1 < nsteps:
                stop = max(float(e.ctx.dev_poll()[1]) for e in self.engines)
                if self.comm.allreduce(stop, "max") > 0.0:
                    break
        polls = [e.ctx.dev_poll() for e in self.engines]
        if overlap:
            for e in self.engines:
                e.set_halo_stream(None)
        code = max(float(st) for st, _, _, _ in polls)
        code = int(self.comm.allreduce(code, "max"))
        self.time = polls[0][2]
        self.steps = polls[0][3]
        return code

    def run(self, nsteps: int, check_every: int = 1) -> int:
        """nsteps steps with stop_sim's checks (IO_rot.f90:625-674) every check_every steps:
        returns 0, 3 (NaN) or 4 (dt <= 1e-12), the same on every rank."""
        for n in range(nsteps):
            dt = self.step()
            if dt <= 1.0e-12:
                return 4
            if (n + 1) % check_every == 0 or n == nsteps - 1:
                bad = max(float(e.has_nan()) for e in self.engines)
                if self.comm.allreduce(bad, "max") > 0.0:
                    return 3
        return 0

    def write_output(self, outdir: str, nout: int, s_global) -> None:
        """output() of the decomposed state (IO_rot.f90:39-105): rank 0 creates the file of
        the global grid, then every rank writes its block's hyperslab (pip_b200.output)."""
        from . import output
        if self.comm.rank == 0:
            output.create_output(outdir, nout, s_global, self.time)
        self.comm.barrier()
        for e in self.engines:
            U_h, U_m = e.download()
            ac = e.alpha_c() if s_global.flag_col >= 2 else None
            output.write_output_block(outdir, nout, s_global, e.block, U_h, U_m, ac)
        self.comm.barrier()

    def close(self) -> None:
        for e in self.engines:
            e.close()
