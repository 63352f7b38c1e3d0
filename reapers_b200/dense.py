"""Exact diagonalisation for small states: the reference's
EvolutionAlgorithm::ExactDiagonalization (inc/algo.h:27-54) with its matrix
exponential cache (MatexpCache, inc/cpuimpl.h:29-88), on the GPU through the
library's dense path (rp_dense_*, the role of DevSumOps::get_eigensystem and
_matexp, inc/gpuimpl.h:1180-1263).

The dense matrix of H is written on the device from the term table (column m
holds c (-1)^popc(z & m) in row m ^ x for every term), its eigensystem comes
from the library eigensolver (heevd, in the Hamiltonian's precision), and
exp(c H) = V diag(exp(c lambda)) V^H from a scaling kernel and one GEMM; each
exponential is cached under its exponent c with a hit count, and the least
used entry is evicted when the cache would exceed its byte budget (16 GiB
by default, the reference's default).  evolve(psi, t, beta) multiplies psi by
exp(-(beta + i t) H) with the library's dense matrix-vector kernel.  This path
is for small states (the matrix has 4^len entries): 2^12 basis states ->
256 MiB in FP64.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

__all__ = ["DenseEvolver"]


class DenseEvolver:
    def __init__(self, ham, cache_bytes=16 << 30):
        if ham.len > 14:
            raise ValueError("the dense path is for at most 14 qubits (a 4 GiB FP64 matrix)")
        self.ham = ham
        self.cache_bytes = int(cache_bytes)
        self._d = None
        self._evals = None
        self._cache = {}        # (re c, im c) -> [matrix, hits]
        self._size = 0

    @property
    def dtype(self):
        import torch
        from . import RP_C64
        return torch.complex64 if self.ham.dtype == RP_C64 else torch.complex128

    def _system(self):
        from . import _lib
        if self._d is None:
            b = np.ascontiguousarray(self.ham.bits, dtype=np.uint64)
            c = np.ascontiguousarray(self.ham.coeff, dtype=np.complex128).view(np.float64)
            d = C.c_void_p()
            _lib.call("rp_dense_create", C.byref(d), self.ham.len, self.ham.dtype, len(b),
                      b.ctypes.data_as(C.POINTER(C.c_uint64)),
                      c.ctypes.data_as(C.POINTER(C.c_double)))
            self._d = d
            ev = np.zeros(1 << self.ham.len)
            _lib.call("rp_dense_eigenvalues", d, ev.ctypes.data_as(C.POINTER(C.c_double)))
            self._evals = ev
        return self._d

    def eigenvalues(self):
        """Eigenvalues of the Hermitian H, ascending (FP64 copy)."""
        self._system()
        return self._evals

    def eigenvectors(self):
        """The eigenvectors as the columns of a (2^len, 2^len) device tensor."""
        import torch
        from . import _lib, _ptr
        D = 1 << self.ham.len
        p = C.c_void_p()
        _lib.call("rp_dense_eigenvectors", self._system(), C.byref(p))
        flat = torch.empty(D * D, dtype=self.dtype, device="cuda")
        _lib.call("rp_memcpy", _ptr(flat), p, flat.numel() * flat.element_size(), 2)
        return flat.view(D, D).T          # column-major storage: [i, j] = V_ij

    def eigenvector(self, index):
        """Eigenvector `index` (ascending order) as a device vector."""
        import torch
        from . import _lib, _ptr
        out = torch.empty(1 << self.ham.len, dtype=self.dtype, device="cuda")
        _lib.call("rp_dense_eigenvector", self._system(), int(index), _ptr(out))
        return out

    def matexp(self, c):
        """exp(c H) as a dense column-major device matrix (a flat tensor of
        4^len elements), cached under c (HostSumOps::matexp and MatexpCache)."""
        import torch
        from . import _lib, _ptr
        key = (float(np.real(c)), float(np.imag(c)))
        hit = self._cache.get(key)
        if hit is not None:
            hit[1] += 1
            return hit[0]
        D = 1 << self.ham.len
        E = torch.empty(D * D, dtype=self.dtype, device="cuda")
        _lib.call("rp_dense_expm", self._system(), key[0], key[1], _ptr(E))
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
        import torch
        from . import _lib, _ptr, _tcode
        if psi.dtype != self.dtype or psi.numel() != 1 << self.ham.len:
            raise ValueError(f"state must be {self.dtype} of length {1 << self.ham.len}, "
                             f"got {psi.dtype} of length {psi.numel()}")
        if t == 0.0 and beta == 0.0:
            return psi
        E = self.matexp(complex(-beta, -t))
        out = torch.empty_like(psi)
        _lib.call("rp_mat_vec", _tcode(psi), psi.numel(), _ptr(E), _ptr(psi), _ptr(out))
        psi.copy_(out)
        return psi

    def ground_state(self):
        """(lowest eigenvalue, its eigenvector) (ExactDiagonalization::ground_state)."""
        return float(self.eigenvalues()[0]), self.eigenvector(0)

    def cache_info(self):
        return {"entries": len(self._cache), "bytes": self._size,
                "hits": {k: v[1] for k, v in self._cache.items()}}

    def close(self):
        from . import _lib
        self._cache = {}
        self._size = 0
        if self._d is not None:
            _lib.load().rp_dense_destroy(self._d)
            self._d = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
