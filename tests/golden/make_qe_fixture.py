"""Generate tests/golden/qe_si.npz from the reference's QE test data
test/example3 (fcc Si, 16^3 grid, 6 bands, 3 irreducible k-points expanded to
the 8-point mesh by 48 space-group operations, half of them with the
fractional translation (1/4, 1/4, 1/4)).  test/example1 (HF) and
test/example3 (BITC) start from the same QE files.

The files hold what tc_b200.qe.QEData reads from data-file-schema.xml and
wfc{1,2,3}.dat_nonbin (cell, FFT grid, symmetry operations, k-points, Miller
indices, coefficients, occupations), so the tests run without the reference
tree.  Run from the repository root, with the reference checked out:

    python tests/golden/make_qe_fixture.py /path/to/TC/test
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tc_b200.qe import QEData  # noqa: E402


def main(test_dir):
    q = QEData(os.path.join(test_dir, "example3"))
    out = os.path.join(HERE, "qe_si.npz")
    q.save_npz(out)
    print(out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/test")
