"""Closed-shell SCF of many molecules at once, the whole iteration on the GPU.

The reference runs one molecule at a time: pyscf.scf.hf.kernel
(pyscf/scf/hf.py:47-242) with get_fock (:1077-1125) and CDIIS
(pyscf/scf/diis.py:40-66, pyscf/lib/diis.py:202-274), eig (:1340) and
make_rdm1 (:840) on the host.  Here one iteration of every molecule of a
batch is:

  1. J/K of all molecules in one batched build (b200jk_batch_get_jk_async:
     one launch per quartet class over a global quartet queue);
  2. Fock F = h + J - K/2 and energy E = E_nuc + 1/2 tr(D (h + F)), batched
     over the molecules padded to the largest basis;
  3. commutator DIIS on F with the error X^T (F D S - S D F) X (the DIIS
     system solved for all molecules at once, with no host synchronisation);
  4. the new density from the orthogonalised Fock matrix F' = X^T F X
     (X = S^{-1/2}) by canonical purification (Palser and Manolopoulos,
     Phys. Rev. B 58, 12704 (1998)): matrix products converging to the
     projector onto the lowest nocc eigenvectors, which is what make_rdm1 of
     the aufbau occupation builds from eig; D = 2 X P X^T.

Every step is a fixed sequence of kernels on device tensors, so one
iteration of the whole batch is captured once as a CUDA graph and replayed.
The padding of each molecule to the largest basis is an identity in S and a
level far above the virtual spectrum in h, so padded states stay empty.
The initial density is the core-Hamiltonian guess (the reference's default
is minao, hf.py:347-474, which is not built here); the converged energy does
not depend on it.  One-electron integrals come from the GPU
(b200jk_int1e).
"""
import numpy

from . import lib

PAD_LEVEL = 50.0     # Eh, diagonal of h (and F) on the padded orbitals


class BatchRHF:
    def __init__(self, plans, nelec, e_nuc, diis_space=6, purify_steps=40):
        import torch
        self.torch = torch
        self.plans = list(plans)
        self.B = len(self.plans)
        dev = torch.device('cuda', self.plans[0].device)
        self.dev = dev
        f64 = torch.float64
        self.nao = [p.nao for p in self.plans]
        N = max(self.nao)
        self.N = N
        self.nocc = torch.tensor([int(n) // 2 for n in nelec], device=dev, dtype=f64)
        self.e_nuc = torch.tensor(numpy.asarray(e_nuc, dtype=float), device=dev, dtype=f64)
        self.m = int(diis_space)
        self.purify_steps = int(purify_steps)
        # flat per-molecule buffers (the batched build reads and writes
        # C-contiguous (nao, nao) arrays), one zero slot at the end for the
        # padded positions of the gathers
        sizes = [n * n for n in self.nao]
        offs = numpy.concatenate([[0], numpy.cumsum(sizes)])
        total = int(offs[-1])
        self.Dflat = torch.zeros(total + 1, device=dev, dtype=f64)
        self.Jflat = torch.zeros(total + 1, device=dev, dtype=f64)
        self.Kflat = torch.zeros(total + 1, device=dev, dtype=f64)
        view = lambda buf, m: buf[offs[m]:offs[m + 1]].view(self.nao[m], self.nao[m])  # noqa: E731
        self.Dm = [view(self.Dflat, m) for m in range(self.B)]
        self.Jm = [view(self.Jflat, m) for m in range(self.B)]
        self.Km = [view(self.Kflat, m) for m in range(self.B)]
        gidx = numpy.full((self.B, N, N), total, dtype=numpy.int64)
        mask = numpy.zeros((self.B, N, N), dtype=bool)
        for m, n in enumerate(self.nao):
            gidx[m, :n, :n] = offs[m] + numpy.arange(n * n).reshape(n, n)
            mask[m, :n, :n] = True
        self.gidx = torch.tensor(gidx, device=dev)
        self.mask = torch.tensor(mask, device=dev)
        self.pad_pos = torch.nonzero(self.mask.reshape(-1), as_tuple=False).reshape(-1)
        self.flat_pos = self.gidx.reshape(-1)[self.pad_pos]
        # one-electron integrals (GPU), padded
        S = torch.zeros((self.B, N, N), device=dev, dtype=f64)
        H = torch.zeros((self.B, N, N), device=dev, dtype=f64)
        eye = torch.eye(N, device=dev, dtype=f64)
        for m, p in enumerate(self.plans):
            n = self.nao[m]
            s, h = p.int1e(device=True)
            S[m, :n, :n] = s
            H[m, :n, :n] = h
            S[m, n:, n:] = eye[n:, n:]
            H[m, n:, n:] = PAD_LEVEL * eye[n:, n:]
        self.S, self.H = S, H
        w, v = torch.linalg.eigh(S)
        self.X = v @ torch.diag_embed(w.rsqrt()) @ v.transpose(1, 2)
        # DIIS history and the state of the iteration
        self.Fh = torch.zeros((self.B, self.m, N, N), device=dev, dtype=f64)
        self.Eh = torch.zeros((self.B, self.m, N, N), device=dev, dtype=f64)
        self.count = torch.zeros((), device=dev, dtype=torch.int64)
        self.D = torch.zeros((self.B, N, N), device=dev, dtype=f64)
        self.energy = torch.zeros(self.B, device=dev, dtype=f64)
        self.energy_last = torch.zeros(self.B, device=dev, dtype=f64)
        self.idem_err = torch.zeros(self.B, device=dev, dtype=f64)
        self.batch = lib.Batch(self.plans)
        self.graph = None

    # -- pieces of one iteration -------------------------------------------
    def _density_from(self, F):
        """D = 2 X P X^T, P the purified projector of F' = X^T F X."""
        torch = self.torch
        Fo = self.X.transpose(1, 2) @ F @ self.X
        N = self.N
        diag = torch.diagonal(Fo, dim1=1, dim2=2)
        off = Fo.abs().sum(dim=2) - diag.abs()
        emin = (diag - off).min(dim=1).values
        emax = (diag + off).max(dim=1).values
        mu = diag.sum(dim=1) / N
        ne = self.nocc
        lam = torch.minimum(ne / (emax - mu), (N - ne) / (mu - emin))
        eye = torch.eye(N, device=self.dev, dtype=Fo.dtype)
        P = (lam / N)[:, None, None] * (mu[:, None, None] * eye - Fo) + (ne / N)[:, None, None] * eye
        for _ in range(self.purify_steps):
            P2 = P @ P
            P3 = P2 @ P
            tr_p = torch.diagonal(P, dim1=1, dim2=2).sum(1)
            tr_p2 = torch.diagonal(P2, dim1=1, dim2=2).sum(1)
            tr_p3 = torch.diagonal(P3, dim1=1, dim2=2).sum(1)
            den = tr_p - tr_p2
            live = den.abs() > 1e-13
            c = torch.where(live, (tr_p2 - tr_p3) / torch.where(live, den, torch.ones_like(den)),
                            torch.full_like(den, 0.5))
            c3 = c[:, None, None]
            up = ((1 + c3) * P2 - P3) / c3
            lo = ((1 - 2 * c3) * P + (1 + c3) * P2 - P3) / (1 - c3)
            Pn = torch.where((c >= 0.5)[:, None, None], up, lo)
            P = torch.where(live[:, None, None], Pn, P)
        self.idem_err.copy_((P @ P - P).abs().amax(dim=(1, 2)))
        return 2.0 * (self.X @ P @ self.X.transpose(1, 2))

    def _fock(self):
        torch = self.torch
        self.batch.get_jk_device_async(self.Dm, self.Jm, self.Km, hermi=1)
        J = torch.take(self.Jflat, self.gidx)
        K = torch.take(self.Kflat, self.gidx)
        return self.H + J - 0.5 * K

    def _diis(self, F):
        torch = self.torch
        err = F @ self.D @ self.S
        err = err - err.transpose(1, 2)
        err = self.X.transpose(1, 2) @ err @ self.X
        slot = torch.remainder(self.count, self.m).reshape(1)
        self.Fh.index_copy_(1, slot, F[:, None])
        self.Eh.index_copy_(1, slot, err[:, None])
        self.count += 1
        nvalid = torch.clamp(self.count, max=self.m)
        valid = torch.arange(self.m, device=self.dev) < nvalid
        Bm = torch.einsum('bipq,bjpq->bij', self.Eh, self.Eh)
        scale = torch.diagonal(Bm, dim1=1, dim2=2).amax(dim=1).clamp(min=1e-300)
        Bm = Bm / scale[:, None, None]
        vv = (valid[:, None] & valid[None, :]).to(Bm.dtype)
        eye = torch.eye(self.m, device=self.dev, dtype=Bm.dtype)
        Bm = Bm * vv + eye * (1 - vv)
        A = torch.zeros((self.B, self.m + 1, self.m + 1), device=self.dev, dtype=Bm.dtype)
        A[:, :self.m, :self.m] = Bm
        vd = valid.to(Bm.dtype)
        A[:, :self.m, self.m] = -vd
        A[:, self.m, :self.m] = -vd
        rhs = torch.zeros((self.B, self.m + 1, 1), device=self.dev, dtype=Bm.dtype)
        rhs[:, self.m, 0] = -1.0
        c, _ = torch.linalg.solve_ex(A, rhs)
        c = c[:, :self.m, 0] * vd
        return torch.einsum('bi,bipq->bpq', c, self.Fh)

    def _set_density(self, D):
        self.D.copy_(D)
        self.Dflat.index_put_((self.flat_pos,), D.reshape(-1)[self.pad_pos])

    def step(self):
        """One SCF iteration of every molecule (capturable)."""
        F = self._fock()
        self.energy_last.copy_(self.energy)
        self.energy.copy_(self.e_nuc + 0.5 * ((self.D * (self.H + F)) * self.mask).sum(dim=(1, 2)))
        Fd = self._diis(F)
        self._set_density(self._density_from(Fd))

    # -- driver ---------------------------------------------------------------
    def start(self):
        """Core-Hamiltonian guess, buffers sized by one synchronous build."""
        self._set_density(self._density_from(self.H))
        self.batch.get_jk_device(self.Dm, hermi=1)
        self.torch.cuda.synchronize(self.dev)

    def capture(self):
        """Record one iteration as a CUDA graph (after start())."""
        torch = self.torch
        side = torch.cuda.Stream(self.dev)
        side.wait_stream(torch.cuda.current_stream(self.dev))
        # the state after a warm-up iteration on the side stream is the
        # state the graph continues from
        with torch.cuda.stream(side):
            self.step()
        torch.cuda.current_stream(self.dev).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.step()
        self.torch.cuda.synchronize(self.dev)

    def run(self, iterations, use_graph=True):
        for _ in range(iterations):
            if use_graph and self.graph is not None:
                self.graph.replay()
            else:
                self.step()
        self.torch.cuda.synchronize(self.dev)
        return self.energy.cpu().numpy(), (self.energy - self.energy_last).abs().cpu().numpy()
