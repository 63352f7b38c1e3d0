"""Library context lifecycle: rp_shutdown followed by rp_init.

rp_shutdown frees the library's streams, workspaces and lazily allocated
scratch (the one-off inner product's and norm's per-CTA partials, the
step-size candidates' expm buffer); a later rp_init on the same device
allocates them afresh, and results stay correct.  A process stays bound to
its first device: rp_init on another one is refused before any CUDA call.
Run in a child process so the shutdown does not disturb the other tests'
library state.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import reapers_b200 as rb
from reapers_b200 import _lib
lib = _lib.load()
rng = np.random.default_rng(5)
n = (1 << 20) + 3
a = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).cuda()
b = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).cuda()
ref = np.vdot(a.cpu().numpy(), b.cpu().numpy())
for rnd in range(3):
    rb.init(0)
    got = rb.dot(a, b)
    assert abs(got - ref) <= 1e-12 * abs(ref), (rnd, got, ref)
    nrm = rb.norm(a)
    assert abs(nrm - np.linalg.norm(a.cpu().numpy())) <= 1e-12 * nrm
    H = np.zeros((4, 4), dtype=np.complex128)
    H[0, 1] = H[1, 0] = 1.0
    fr = np.array([0.0, 1.0]); fi = np.array([-0.5, 0.0])
    col = np.zeros((2, 4), dtype=np.complex128)
    assert lib.rp_expm_first_column(4, H.T.copy().ctypes.data_as(C.POINTER(C.c_double)), 2,
        fr.ctypes.data_as(C.POINTER(C.c_double)), fi.ctypes.data_as(C.POINTER(C.c_double)),
        col.ctypes.data_as(C.POINTER(C.c_double))) == 0, lib.rp_last_error()
    assert abs(col[0, 0] - np.cos(0.5)) < 1e-14 and abs(col[0, 1] + 1j * np.sin(0.5)) < 1e-14
    assert lib.rp_shutdown() == 0
rc = lib.rp_init(1)
assert rc == -2, rc
assert b"bound to device 0" in lib.rp_last_error()
rb.init(0)
print("lifecycle ok")
"""


def test_shutdown_then_init_reallocates_scratch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "lifecycle ok" in r.stdout
