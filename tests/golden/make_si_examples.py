"""Generate the fixtures of the golden-replay tests from the reference's test
data test/example1 (HF), test/example2 (TC) and test/example3 (BITC): fcc Si,
16^3 grid, 6 bands, 3 irreducible k-points expanded to 8 by symmetry, all
three starting from the same Quantum ESPRESSO files.

  qe_si.npz        the QE data TC++ reads (tc_b200.qe.QEData.save_npz, with atoms)
  si_upf.npz       the arrays TC++ reads from Si_test.upf (tc_b200.upf.UPF)
  si_examples.json per example: calc_method, the RPA F of parameters.casl, and
                   the energies TC++ printed after SCF iterations 1 and 2
                   ("Total energy (1-body terms)" and so on, output.out), with
                   the orbital energies (eV) printed after iteration 1

Run from the repository root, with the reference checked out:

    python tests/golden/make_si_examples.py /path/to/TC/test
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tc_b200.qe import QEData  # noqa: E402
from tc_b200.upf import read_casl_rpa, read_upf  # noqa: E402

EXAMPLES = {"example1": "HF", "example2": "TC", "example3": "BITC"}


def parse_output(path):
    """Energies of every SCF iteration and orbital energies after the first."""
    text = open(path).read()
    num = r"([-+0-9.eE]+)"
    cplx = r"\(\s*" + num + r"\s*,\s*" + num + r"\s*\)"
    iters = []
    for block in re.split(r"\n Iteration \d+\n", text)[1:]:
        e = {}
        for key in ("1-body", "2-body", "3-body"):
            m = re.search(r"Total energy \(" + key + r" terms\) = " + cplx, block)
            if m:
                e[key] = [float(m.group(1)), float(m.group(2))]
        m = re.search(r"Total energy \(Ewald energy\) = " + num, block)
        if m:
            e["ewald"] = float(m.group(1))
        bands = []
        for kb in re.finditer(r"k-vector([^\n]*)\n\s*\(band index, energy \(eV\), filling\)\n((?:\s*\d+ [^\n]+\n)+)",
                              block):
            bands.append([float(line.split()[1]) for line in kb.group(2).strip().split("\n")])
        if e:
            e["orbital_energies_eV"] = bands
            iters.append(e)
    return iters


def main(test_dir):
    q = QEData(os.path.join(test_dir, "example1"))
    q.save_npz(os.path.join(HERE, "qe_si.npz"))
    upf = read_upf(os.path.join(test_dir, "example1", "Si_test.upf"))
    np.savez_compressed(os.path.join(HERE, "si_upf.npz"), **upf.arrays())
    out = {}
    for ex, method in EXAMPLES.items():
        d = os.path.join(test_dir, ex)
        rec = {"calc_method": method, "iterations": parse_output(os.path.join(d, "output.out"))}
        casl = os.path.join(d, "parameters.casl")
        if os.path.exists(casl):
            rec["F"] = read_casl_rpa(casl)[1].tolist()
        out[ex] = rec
    with open(os.path.join(HERE, "si_examples.json"), "w") as f:
        json.dump(out, f, indent=1)
    for ex, rec in out.items():
        print(ex, rec["calc_method"], rec.get("F"), rec["iterations"][0].get("2-body"))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/test")
