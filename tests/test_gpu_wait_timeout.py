"""The failure path of the row kernel's pipeline waits, driven on the GPU
without a fault: a barrier whose expected copy never arrives.

rp_test_withhold_tile makes the next row-kernel launch withhold one tile copy
in its first CTA, so that CTA's consumers wait on a barrier that nothing
completes.  Every wait is bounded: the consumers give up, the producer's
wait for the released stage gives up, the CTA lets its copies in flight land
and returns.  The host then reads RP_E_DEVICE from the launch's error word
(rp_synchronize, like the reference's error peek in GPUImpl::sync_device,
inc/gpuimpl.h:634-638) and the context stays usable: the next apply is
correct.  The other CTAs' output tiles are complete.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POLLS = 1 << 16   # the first CTA's wait limit in the test (polls); the default is 2^26


@pytest.mark.parametrize("dtype,L", [("c64", 20), ("c128", 19)])
@pytest.mark.parametrize("iteration", [0, 3])
def test_withheld_tile_gives_device_error_then_recovers(cuda, dtype, L, iteration):
    import torch
    import reapers_b200 as rb
    from reapers_b200 import _lib
    bits, coeff = rb.syk.sparse_syk(2 * L, k=8, seed=11)
    ham = rb.Hamiltonian(L, bits, coeff, dtype)
    info = ham.info()
    assert info["kernel"] == 2, "the row kernel must be the one planned"
    x = rb.random_state(L, dtype, seed=4)
    good = torch.empty_like(x)
    ham.apply(good, x)
    rb.synchronize()
    y = torch.zeros_like(x)
    _lib.call("rp_test_withhold_tile", iteration, POLLS)
    ham.apply(y, x)   # asynchronous: returns before the waits give up
    with pytest.raises(rb.RPError) as e:
        rb.synchronize()
    assert e.value.code == -5
    assert "gave up" in str(e.value)
    # the report is cleared once read
    rb.synchronize()
    # every output tile of the other CTAs was written; the first CTA's first
    # tile was not finished (its rows were never stored)
    tile = 1 << info["tile_exp"]
    grid = info["window"]
    yc, gc = y.cpu().numpy(), good.cpu().numpy()
    mask = np.ones(1 << L, bool)
    for t in range(0, (1 << L) // tile, grid):
        mask[t * tile:(t + 1) * tile] = False
    assert np.array_equal(yc[mask], gc[mask])
    assert not np.array_equal(yc[:tile], gc[:tile])
    # the context is usable and the next product is correct (bit-identical)
    z = torch.empty_like(x)
    ham.apply(z, x)
    rb.synchronize()
    assert torch.equal(z, good)
    ham.close()


def test_withhold_arguments_are_checked(cuda):
    import reapers_b200 as rb
    from reapers_b200 import _lib
    with pytest.raises(rb.RPError):
        _lib.call("rp_test_withhold_tile", -1, POLLS)
    with pytest.raises(rb.RPError):
        _lib.call("rp_test_withhold_tile", 0, 10)
