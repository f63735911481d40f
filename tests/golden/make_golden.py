"""Generate the golden tau00 fixtures from the reference's own C++ path.

Runs oracle/_ref/libtauref.so (the reference's calculateTauMatrix compiled from its source tree by
oracle/Makefile) on seeded inputs from lsms_b200.workloads and stores, per case, the tau00_l the
reference returns for solver ids 0x2005 (zblocklu_cpp) and 0x2001 (zgesv), a checksum of the inputs
(so a drift of the input generator is caught), and row/column sums of the reference's KKR matrix.

    python tests/golden/make_golden.py      # needs the reference tree to build the oracle
"""

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from lsms_b200 import workloads as W  # noqa: E402
from oracle import reflib  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def cases():
    """name -> (problem factory, list of (iie, ispin))."""
    return {
        "bcc15_E0.6": (lambda: W.config_small(), [(0, 0)]),
        "bcc15_Em0.2": (lambda: W.make_problem("bcc", 5.42, 2, 3, [-0.2 + 0.1j], 11, n_species=1), [(0, 0)]),
        "bcc15_contour": (lambda: W.make_problem("bcc", 5.42, 2, 3, W.semicircle_contour(-0.3, 0.7, 4), 12,
                                                 n_species=2), [(0, 0), (1, 0), (2, 0), (3, 0)]),
        "bcc15_noncollinear": (lambda: W.make_problem("bcc", 5.42, 2, 3, [0.5 + 0.05j], 13, n_species=None,
                                                      n_spin_cant=2, n_spin_pola=2), [(0, 0)]),
        "bcc15_polarized": (lambda: W.make_problem("bcc", 5.42, 2, 3, [0.45 + 0.02j], 14, n_species=2,
                                                   n_spin_pola=2), [(0, 0), (0, 1)]),
        "bcc15_lmax_steps": (lambda: W.make_problem("bcc", 5.42, 2, 3, [0.55 + 0.03j], 15, n_species=2,
                                                    liz_lmax=[3] * 9 + [2] * 6), [(0, 0)]),
        "fcc43_E0.3": (lambda: W.make_problem("fcc", 6.82, 3, 3, [0.3 + 0.1j], 16, n_species=2), [(0, 0)]),
    }


def input_digest(prob) -> str:
    h = hashlib.sha256()
    for a in (prob.liz_pos, prob.liz_lmax, prob.liz_store_idx, prob.tmat_store, prob.energies):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    for name, (make, runs) in cases().items():
        prob = make()
        out = {"digest": np.array(input_digest(prob))}
        for iie, ispin in runs:
            tag = f"{iie}_{ispin}"
            out[f"tau_blocklu_{tag}"] = reflib.calculate_tau(prob, iie, ispin, reflib.ZBLOCKLU_CPP)
            out[f"tau_zgesv_{tag}"] = reflib.calculate_tau(prob, iie, ispin, reflib.ZGESV)
            m = reflib.build_kkr(prob, iie, ispin)
            out[f"m_rowsum_{tag}"] = m.sum(1)
            out[f"m_colsum_{tag}"] = m.sum(0)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, prob.nrmat_ns, len(runs))


if __name__ == "__main__":
    main()
