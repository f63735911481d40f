"""Seeded input generator: geometry and layouts match the reference's conventions."""

import numpy as np

from lsms_b200 import workloads as W


def test_shell_counts():
    assert W.lattice_shells("bcc", 5.42, 2).shape == (3, 15)
    assert W.lattice_shells("fcc", 6.82, 7).shape == (3, 135)
    sizes = [W.lattice_shells("fcc", 6.82, s).shape[1] for s in (3, 4, 5, 6, 7)]
    assert sizes == [43, 55, 79, 87, 135]


def test_central_site_first_and_sorted():
    p = W.lattice_shells("fcc", 6.82, 7)
    d = np.sqrt((p ** 2).sum(0))
    assert d[0] == 0 and np.all(np.diff(d) >= -1e-12)


def test_n2160_config_sizes():
    prob = W.config_n2160()
    assert prob.nrmat_ns == 2160 and prob.kkrsz_ns == 16 and prob.energies.size == 31
    assert prob.tmat_store.shape == (2, 31, 1024)


def test_contour_on_semicircle():
    e = W.semicircle_contour(-0.3, 0.7, 31)
    assert np.allclose(np.abs(e - 0.2), 0.5)
    assert np.all(e.imag > 0)


def test_t_matrix_layout_noncollinear():
    prob = W.make_problem("bcc", 5.42, 2, 3, [0.5 + 0.05j], 3, n_species=None, n_spin_cant=2, n_spin_pola=2)
    t = prob.t_block(0, 0)
    assert t.shape == (32, 32)
    # the spin rotation is unitary: eigenvalues of t are the collinear t_l values
    ev = np.sort_complex(np.linalg.eigvals(t))
    assert np.all(np.isfinite(ev))
