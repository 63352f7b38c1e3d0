"""Exact diagonalisation for small states: the reference's
EvolutionAlgorithm::ExactDiagonalization (inc/algo.h:27-54) with its matrix
exponential cache (MatexpCache, inc/cpuimpl.h:29-88), on the GPU.

The dense matrix of H is built column by column with the library's H.psi
kernel (column j = H e_j), its eigensystem by cuSOLVER (through
torch.linalg.eigh, FP64 or FP32 as the Hamiltonian), and exp(c H) =
V diag(exp(c lambda)) V^H by cuBLAS GEMMs; each exponential is cached under
its exponent c with a hit count, and the least used entry is evicted when
the cache would exceed its byte budget (16 GiB by default, the reference's
default).  evolve(psi, t, beta) multiplies psi by exp(-(beta + i t) H); the
reference's dense fallback for #terms >= 2^len (inc/cpuimpl.h:742) uses the
same matrix.  This path is for small states (the matrix has 4^len entries):
2^12 basis states -> 256 MiB in FP64.
"""
from __future__ import annotations

import numpy as np

__all__ = ["DenseEvolver"]


class DenseEvolver:
    def __init__(self, ham, cache_bytes=16 << 30):
        if ham.len > 14:
            raise ValueError("the dense path is for at most 14 qubits (a 4 GiB FP64 matrix)")
        self.ham = ham
        self.cache_bytes = int(cache_bytes)
        self._M = None
        self._eig = None
        self._cache = {}        # (re c, im c) -> [matrix, hits]
        self._size = 0

    @property
    def dtype(self):
        import torch
        from . import RP_C64
        return torch.complex64 if self.ham.dtype == RP_C64 else torch.complex128

    def matrix(self):
        """The dense matrix of H (column j = H e_j), built once."""
        import torch
        if self._M is None:
            D = 1 << self.ham.len
            M = torch.empty((D, D), dtype=self.dtype, device="cuda")
            e = torch.zeros(D, dtype=self.dtype, device="cuda")
            col = torch.empty(D, dtype=self.dtype, device="cuda")
            for j in range(D):
                e[j] = 1
                self.ham.apply(col, e)
                M[:, j] = col
                e[j] = 0
            torch.cuda.synchronize()
            self._M = M
        return self._M

    def eigensystem(self):
        """(eigenvalues ascending, eigenvectors as columns) of the Hermitian H."""
        import torch
        if self._eig is None:
            self._eig = torch.linalg.eigh(self.matrix())
        return self._eig

    def matexp(self, c):
        """exp(c H), cached under c (HostSumOps::matexp and MatexpCache)."""
        import torch
        key = (float(np.real(c)), float(np.imag(c)))
        hit = self._cache.get(key)
        if hit is not None:
            hit[1] += 1
            return hit[0]
        lam, V = self.eigensystem()
        f = torch.exp(complex(c) * lam.to(self.dtype))
        E = (V * f) @ V.conj().T
        nbytes = E.numel() * E.element_size()
        while self._cache and self._size + nbytes > self.cache_bytes:
            victim = min(self._cache, key=lambda k: self._cache[k][1])
            self._size -= self._cache[victim][0].numel() * self._cache[victim][0].element_size()
            del self._cache[victim]
        self._cache[key] = [E, 0]
        self._size += nbytes
        return E

    def evolve(self, psi, t, beta=0.0):
        """psi <- exp(-(beta + i t) H) psi in place (ExactDiagonalization::evolve)."""
        if t == 0.0 and beta == 0.0:
            return psi
        psi.copy_(self.matexp(complex(-beta, -t)) @ psi)
        return psi

    def ground_state(self):
        """(lowest eigenvalue, its eigenvector) (ExactDiagonalization::ground_state)."""
        lam, V = self.eigensystem()
        return float(lam[0]), V[:, 0].contiguous()

    def cache_info(self):
        return {"entries": len(self._cache), "bytes": self._size,
                "hits": {k: v[1] for k, v in self._cache.items()}}
