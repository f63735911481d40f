"""The C++ adapter include/b200tau_lsms_adapter.hpp: compiles against stand-ins of the LSMS types
(always) and against the reference's own headers (when the reference tree is present), and on a GPU
gives the reference's tau00 through calculateTauMatrix_b200 / calculateAllTauMatrices_b200."""

import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the reference tree, as oracle/Makefile reads it (REF, with the same default)
REF = os.environ.get("REF", "/root/reference")
LIBDIR = os.path.join(ROOT, "lsms_b200", "_lib")


def build_driver(outdir: str) -> str:
    exe = os.path.join(outdir, "adapter_driver")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(ROOT, "tests", "adapter"), os.path.join(ROOT, "tests", "adapter", "adapter_driver.cpp"),
           "-L", LIBDIR, "-lb200tau", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-3000:]
    return exe


def test_adapter_builds_with_stand_in_types(tmp_path):
    build_driver(str(tmp_path))


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src", "MultipleScattering")),
                    reason="reference tree not present")
def test_adapter_compiles_against_reference_headers(tmp_path):
    src = tmp_path / "use_ref_types.cpp"
    src.write_text('''
#include "Complex.hpp"
#include "Matrix.hpp"
#include "Main/SystemParameters.hpp"
#include "b200tau_lsms_adapter.hpp"
int use(LSMSSystemParameters &lsms, LocalTypeInfo &local, Complex e, Complex *out, Matrix<Complex> &m,
        Matrix<Complex> &all) {
  int rc = b200tau_lsms::uploadTmatStore_b200(lsms, local);
  rc |= b200tau_lsms::setAtoms_b200(lsms, local);
  rc |= b200tau_lsms::calculateTauMatrix_b200(lsms, local, local.atom[0], 0, 0, e, e, out, m, 0);
  rc |= b200tau_lsms::calculateAllTauMatrices_b200(lsms, local, e, 0, all, 1.0e-5);
  return rc;
}
''')
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-w", "-I", os.path.join(ROOT, "oracle", "ref_shim"),
           "-I", os.path.join(REF, "include"), "-I", os.path.join(REF, "src"), "-I",
           os.path.join(REF, "src", "Main"), "-I", os.path.join(REF, "src", "Misc"), "-I",
           os.path.join(REF, "src", "Potential"), "-I", os.path.join(ROOT, "include"), str(src)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-3000:]


@pytest.mark.gpu
def test_adapter_matches_reference(ref, tmp_path):
    from lsms_b200 import workloads as W
    prob = W.make_problem("bcc", 5.42, 2, 3, W.semicircle_contour(-0.3, 0.7, 3), 51, n_species=2)
    exe = build_driver(str(tmp_path))
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([prob.lmax, prob.n_spin_cant, prob.n_spin_pola, prob.num_liz, prob.tmat_store.shape[0],
                  prob.tmat_store.shape[1]], np.int32).tofile(f)
        np.ascontiguousarray(prob.liz_pos.T).tofile(f)
        prob.liz_lmax.astype(np.int32).tofile(f)
        prob.liz_store_idx.astype(np.int32).tofile(f)
        prob.ubr.astype(np.complex128).tofile(f)
        prob.ubrd.astype(np.complex128).tofile(f)
        np.ascontiguousarray(prob.tmat_store).tofile(f)
        prob.energies.astype(np.complex128).tofile(f)
    res = subprocess.run([exe, str(inp), str(outp)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    out = np.fromfile(outp, np.complex128).reshape(4, -1)
    for ie in range(3):
        want = ref.calculate_tau(prob, ie, 0, ref.ZBLOCKLU_CPP)
        t0 = prob.t_block(0, ie).T.reshape(-1)
        assert np.abs(out[ie] - want).max() / np.abs(want + t0).max() <= 1e-12
    assert np.array_equal(out[3], out[0])
