"""A block of a decomposed run on the oracle (CPU): the engine protocol of
pip_b200.decomp (cfl, stage, halo_bytes, message_bytes, buffer, pack, unpack, has_nan,
download, close) with the oracle's orc_stage and its neighbour-aware PIPbnd, and mpi_bnd's
layer slices (MPI_rot.f90:128-339) done on the host arrays.  Message layout: ion planes
then neutral planes, layer, position along the face -- the layout of pip_halo_pack."""
import numpy as np
import torch

from oracle import oracle as O


class OracleBlock:
    def __init__(self, block, U_h, U_m, eta=None):
        self.block = block
        self.s = block.settings
        self.o = O.Oracle(self.s, U_h, U_m)
        self.o.set_neighbors(block.neighbor)
        if eta is not None:
            self.o.set_resistivity(eta)
        ix, jx, _ = self.s.shape
        self.n = (ix, jx)
        self.m = self.s.margin

    def cfl(self):
        return self.o.cfl()

    def stage(self, k, dt, cmax):
        self.o.cmax = cmax
        self.o.stage(k, dt)
        if k == 2 and self.s.flag_heat == 1 and all(n < 0 for n in self.block.neighbor):
            # post_step's conduction and PIPbnd of a block without neighbours, as pip_stage
            self.o.conduction(dt)
            self.o.fill_ghosts()

    def _layers(self, face, pack):
        d = face // 2
        m = self.m[d]
        n = self.n[d]
        lower = face % 2 == 0
        first = (m if lower else n - 2 * m) if pack else (0 if lower else n - m)
        return d, slice(first, first + m)

    def halo_bytes(self, face):
        d = face // 2
        ix, jx = self.n
        return 8 * (self.s.nvar_m + 5) * self.m[d] * (jx if d == 0 else ix)

    def message_bytes(self, face):
        return self.halo_bytes(face)

    def buffer(self, nbytes):
        return torch.empty(nbytes, dtype=torch.uint8)

    def pack(self, face, buf):
        U_h, U_m = self.o.state()
        U = np.concatenate([U_m, U_h], axis=0)
        d, sl = self._layers(face, True)
        msg = U[:, sl, :] if d == 1 else U[:, :, sl].transpose(0, 2, 1)
        raw = np.ascontiguousarray(msg).view(np.uint8).reshape(-1)
        buf[: raw.size] = torch.from_numpy(raw)
        return raw.size

    def unpack(self, face, buf, nbytes):
        U_h, U_m = self.o.state()
        U = np.concatenate([U_m, U_h], axis=0)
        d, sl = self._layers(face, False)
        ix, jx = self.n
        msg = buf[:nbytes].numpy().view(np.float64)
        if d == 1:
            U[:, sl, :] = msg.reshape(U.shape[0], -1, ix)
        else:
            U[:, :, sl] = msg.reshape(U.shape[0], -1, jx).transpose(0, 2, 1)
        nm = self.s.nvar_m
        self.o.set_state(U[nm:], U[:nm])

    # BiCGstabMPI in phases (the engine protocol of DecomposedRun.conduction)
    def hcd_begin(self, dt):
        return self.o.hcd_begin(dt)

    def hcd_phase(self, phase, c0=0.0, c1=0.0):
        return self.o.hcd_phase(phase, c0, c1)

    def hcd_row_bytes(self):
        return 8 * self.n[0]

    def hcd_pack(self, vec, face, buf):
        jx = self.n[1]
        row = self.m[1] if face == 2 else jx - self.m[1] - 1
        raw = self.o.hcd_get_row(vec, row).view(np.uint8)
        buf[: raw.size] = torch.from_numpy(raw.copy())
        return raw.size

    def hcd_unpack(self, vec, face, buf):
        jx = self.n[1]
        row = self.m[1] - 1 if face == 2 else jx - self.m[1]
        self.o.hcd_set_row(vec, row, buf[: 8 * self.n[0]].numpy().view(np.float64))

    def hcd_end(self, iters):
        self.o.hcd_end()
        self.o.fill_ghosts()        # the physical faces; the exchange fills the others

    def stream(self):
        import contextlib
        return contextlib.nullcontext()

    def has_nan(self):
        return self.o.has_nan()

    def download(self):
        return self.o.state()

    def alpha_c(self):
        return self.o.alpha_c()

    def close(self):
        self.o.close()
