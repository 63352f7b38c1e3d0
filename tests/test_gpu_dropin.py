"""The reference's own host code on B200Impl (include/rpb200_impl.hpp).

oracle/_ref/dropin_driver instantiates the reference's State, Krylov, SYK and
FermionOpNonBlockForm templates twice in one process -- on the reference's
CPUImpl and on B200Impl, which routes every backend call through the C ABI
to the sm_100a kernels -- and reports the relative difference of each result:
the SYK term list, the host->device->host state round trip, element access,
State operator* (H.psi), the reference's restarted Krylov evolve, the
GPU-resident Krylov selected as State::evolve<B200Krylov>, imaginary-time
evolution, the OTOC sequence of examples/simple-syk-krylov.cc, an apply
after the operator is changed (device table dropped and rebuilt) or
move-assigned from another (no stale table of the old terms), and the
reference's ground-state Lanczos (energy; state overlap where the ground
state is not degenerate); the reference's exact diagonalisation
(ExactDiagonalization: eigensystem, matexp cache, mat_mul and the
eigenvector copy on the device); and the parity-block form
(FermionOpBlockForm, BlockDiag, BlockState): block term lists, the OTOC
sequence of examples/syk.cc on one block, a block state evolve.
"""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "dropin_driver")


def test_dropin_driver_is_built_against_librpb200():
    assert os.path.exists(DRIVER), "oracle/_ref/dropin_driver was not built"
    out = subprocess.run(["ldd", DRIVER], capture_output=True, text=True).stdout
    line = [ln for ln in out.splitlines() if "librpb200" in ln]
    assert line and "not found" not in line[0], out


@pytest.mark.gpu
@pytest.mark.parametrize("N,sp,seed,t,krydim", [
    (16, 0.0, 3, 1.0, 8),      # dense SYK, 1820 terms >= 2^8: the reference takes its dense path
    (20, 8.0, 5, 2.0, 10),     # sparse SYK k = 8
    (24, 8.0, 7, 1.5, 12),     # sparse SYK, 12 qubits
    (24, 0.0, 1, 1.0, 20),     # dense SYK N = 24 (10626 terms, 12 qubits): the exact
                               # diagonalisation shape of the small-N dense path
])
def test_reference_code_on_b200impl_matches_cpuimpl(N, sp, seed, t, krydim):
    r = subprocess.run([DRIVER, str(N), str(sp), str(seed), str(t), str(krydim)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["term_diff"] == 0.0
    assert d["roundtrip"] == 0.0 and d["elem"] == 0.0
    for k in ("apply", "evolve_ref_krylov", "evolve_b200krylov", "evolve_beta", "mutate", "moved"):
        assert d[k] <= 1e-12, (k, d)
    assert d["otoc"] <= 1e-11, d
    # parity-block form: block gen_ham, the examples/syk.cc OTOC on one block,
    # a BlockState evolved under BlockDiag(H_LL, H_RR)
    assert d["block_terms"] == 0.0
    assert d["otoc_block"] <= 1e-11 and d["block_evolve"] <= 1e-12, d
    # ground state (inc/algo.h:180-257) from different random starts
    assert abs(d["E0_b200"] - d["E0_cpu"]) <= 1e-10 * abs(d["E0_cpu"]), d
    if N % 8 == 0:   # no parity-sector degeneracy: the same state up to a phase
        assert d["ground_overlap"] >= 1 - 1e-8, d
    # exact diagonalisation (inc/algo.h:29-54) on B200Impl: the device
    # eigensystem's ground energy against the CPU backend's Lanczos, the
    # matexp evolve (and its cached repeat, and imaginary time) against the
    # CPU backend's restarted Krylov; up to 2^8 states also against the CPU
    # backend's own exact diagonalisation
    assert abs(d["E0_ed_b200"] - d["E0_cpu"]) <= 1e-9 * abs(d["E0_cpu"]), d
    if N % 8 == 0:
        assert d["ed_overlap"] >= 1 - 1e-8, d
    assert d["ed_evolve"] <= 1e-10 and d["ed_evolve_cached"] <= 1e-10, d
    assert d["ed_cache_bytes"] > 0, d
    assert d["ed_beta"] <= 1e-10, d
    if d["ed_cpu"]:
        assert abs(d["E0_ed_cpu"] - d["E0_ed_b200"]) <= 1e-10 * abs(d["E0_ed_cpu"]), d
        assert d["ed_vs_cpu_ed"] <= 1e-10, d
