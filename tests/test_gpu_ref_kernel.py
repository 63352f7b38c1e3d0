"""The reference's own GPU backend, compiled for sm_100a from its sources
(oracle/_ref/ref_gpu_driver: GPUImpl and its krnl_apply_ops kernel,
src/krnl.cu:81-94, 220-257), as a second, GPU-side baseline: on the same
inputs its H.psi equals the product's row and tiled kernels (FP64 to 1e-12,
FP32 to 1e-5 relative), so timing it beside them compares the same work."""
import os
import subprocess
import tempfile

import numpy as np
import pytest
import torch

import reapers_b200 as rb
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DRIVER = os.path.join(os.path.dirname(O.__file__), "_ref", "ref_gpu_driver")


@pytest.mark.parametrize("L,dtype", [(12, "c128"), (20, "c64"), (20, "c128")])
def test_reference_gpu_kernel_matches_ours(cuda, L, dtype):
    if not os.path.exists(DRIVER):
        pytest.skip("oracle/_ref/ref_gpu_driver was not built")
    bits, coeff = rb.syk.sparse_syk(2 * L, k=8, seed=77)
    rng = np.random.default_rng(5)
    v = rng.standard_normal(1 << L) + 1j * rng.standard_normal(1 << L)
    v /= np.linalg.norm(v)
    tmp = tempfile.mkdtemp(prefix="rpgpu_")
    tf, vf, of = (os.path.join(tmp, n) for n in ("terms", "vec", "out"))
    O.write_terms(tf, L, bits, coeff)
    O.write_vec(vf, v)
    fp = "64" if dtype == "c128" else "32"
    r = subprocess.run([DRIVER, "apply", tf, fp, vf, of], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    ref = O.read_vec(of)
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    tdt = torch.complex128 if dtype == "c128" else torch.complex64
    x = torch.from_numpy(v).to(tdt).cuda()
    y = torch.empty_like(x)
    ham.apply(y, x)
    got = y.cpu().numpy().astype(np.complex128)
    tol = 1e-12 if dtype == "c128" else 1e-5
    assert np.linalg.norm(got - ref) <= tol * np.linalg.norm(ref)
    ham.close()
