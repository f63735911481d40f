"""The oracle is pinned before it is trusted (CPU only).

* Gaunt numbers: the two golden values of the reference's unit test Test/Unit/test_gaunt.cpp:84-87
  (lmax = 3, tolerance 1e-12), for the reference build, the numpy port and the product's table.
* Reference solvers agree with each other (the inversionTest cross-check,
  Test/DevTests/inversionTest/inversionTest.cpp:452-542) and with the committed golden fixtures.
* The numpy port (oracle/port.py) agrees with the reference build on M and tau00.
* Known answers of inversionTest: t = 1, G = 0 gives tau00 = t0 exactly; the Hilbert fixture
  (inversionTest.cpp:88-135) is solved identically by the Schur-complement and the dense solve.
"""

import hashlib
import os

import numpy as np
import pytest

from lsms_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CGNT_000 = 0.28209479177387842
CGNT_166 = 0.1802237515728685748747963944546917104709985754562351930533759359


def test_gaunt_golden_reference(ref):
    cg, illp, ilp1 = ref.tables(3)
    assert abs(cg[0, 0, 0] - CGNT_000) < 1e-12
    assert abs(cg[1, 6, 6] - CGNT_166) < 1e-12
    assert np.allclose(ilp1, [1j ** (l + 1) for l in range(7)], atol=0)


def test_gaunt_golden_port():
    from oracle import port
    _, _, cg, _, _ = port.angular_tables(3)
    assert abs(cg[0, 0, 0] - CGNT_000) < 1e-12
    assert abs(cg[1, 6, 6] - CGNT_166) < 1e-12


def test_gaunt_golden_product():
    from lsms_b200 import tau
    cg = tau.gaunt_numbers(3)
    assert abs(cg[0, 0, 0] - CGNT_000) < 1e-12
    assert abs(cg[1, 6, 6] - CGNT_166) < 1e-12


def test_tables_port_and_product_match_reference(ref):
    from lsms_b200 import tau
    from oracle import port
    cg_ref, illp_ref, ilp1_ref = ref.tables(3)
    _, _, cg_port, illp_port, ilp1_port = port.angular_tables(3)
    cg_prod = tau.gaunt_numbers(3)
    used = cg_port != 0  # the reference leaves entries outside the l3 range unset
    assert np.abs(cg_ref[used] - cg_port[used]).max() < 1e-14
    assert np.abs(cg_ref[used] - cg_prod[used]).max() < 1e-14
    assert np.array_equal(cg_prod != 0, used)
    assert np.abs(illp_ref - illp_port).max() == 0
    assert np.abs(ilp1_ref - ilp1_port).max() == 0


def _golden_cases():
    from tests.golden.make_golden import cases
    return cases()


@pytest.mark.parametrize("name", sorted(__import__("tests.golden.make_golden", fromlist=["cases"]).cases()))
def test_reference_matches_golden(ref, name):
    make, runs = _golden_cases()[name]
    prob = make()
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    from tests.golden.make_golden import input_digest
    assert str(g["digest"]) == input_digest(prob), "input generator drifted from the golden fixture"
    for iie, ispin in runs:
        tag = f"{iie}_{ispin}"
        got = ref.calculate_tau(prob, iie, ispin, ref.ZBLOCKLU_CPP)
        want = g[f"tau_blocklu_{tag}"]
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
        # the reference's own solvers agree (inversionTest cross-check)
        zg = g[f"tau_zgesv_{tag}"]
        assert np.abs(zg - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("name", ["bcc15_E0.6", "bcc15_noncollinear", "bcc15_polarized", "bcc15_lmax_steps"])
def test_port_matches_reference(ref, name):
    from oracle import port
    make, runs = _golden_cases()[name]
    prob = make()
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    for iie, ispin in runs:
        tag = f"{iie}_{ispin}"
        m_port = port.build_kkr(prob, iie, ispin)
        m_ref = ref.build_kkr(prob, iie, ispin)
        assert np.abs(m_port - m_ref).max() <= 1e-13 * np.abs(m_ref).max()
        assert np.abs(m_ref.sum(1) - g[f"m_rowsum_{tag}"]).max() <= 1e-12 * np.abs(m_ref).max()
        tau_port = port.solve(prob, iie, ispin)
        want = g[f"tau_blocklu_{tag}"]
        assert np.abs(tau_port - want).max() <= 1e-12 * np.abs(want).max()


def test_known_answer_identity():
    """inversionTest type 2: t = 1, G = 0 -> M = 1 and tau00 = t0."""
    from oracle import port
    b, nblk = 18, 6
    m = np.eye(b * nblk, dtype=np.complex128)
    t0 = np.eye(b, dtype=np.complex128)
    assert np.array_equal(port.schur_tau00(m, t0), t0)


def hilbert_kkr(b: int, nblk: int) -> tuple[np.ndarray, np.ndarray]:
    """inversionTest type 1 (inversionTest.cpp:88-135): Hilbert t per block and a Hilbert G0 with
    zero diagonal blocks, M = 1 - t G.  (The reference's zeroDiagonalBlocks loop clears every
    block, i.e. G = 0; the intended fixture with only diagonal blocks cleared is used here.)"""
    n = b * nblk
    i = np.arange(n)
    g = 1.0 / (i[:, None] + i[None, :] + 1.0)
    for k in range(nblk):
        g[k * b:(k + 1) * b, k * b:(k + 1) * b] = 0.0
    ib = np.arange(b)
    t = 1.0 / (ib[:, None] + ib[None, :] + 1.0)
    m = np.eye(n, dtype=np.complex128)
    for k in range(nblk):
        m[k * b:(k + 1) * b, :] -= t @ g[k * b:(k + 1) * b, :]
    return m, t.astype(np.complex128)


def test_known_answer_hilbert_crosscheck():
    from oracle import port
    m, t0 = hilbert_kkr(18, 5)
    tau_schur = port.schur_tau00(m, t0)
    rhs = np.zeros((m.shape[0], 18), np.complex128)
    rhs[:18] = t0
    tau_dense = np.linalg.solve(m, rhs)[:18]
    assert np.abs(tau_schur - tau_dense).max() <= 1e-9 * np.abs(tau_dense).max()
