"""Generate the fixtures of the golden-replay tests from the reference's test
data: fcc Si, 16^3 grid, 6 bands per spin, from two Quantum ESPRESSO runs,
each replayed with HF, TC and BITC:

  test/example1-3    3 irreducible k-points (8 by symmetry), fixed occupations
  test/example17-19  spin-polarised (lsda), 3 irreducible k-points, Gaussian smearing (0.1 Ha)
and two Gamma-only QE runs (half of the plane waves stored, 20^3 grid: the
library's runtime-size FFT path) replayed with HF:
  test/example26     unpolarised, fixed occupations
  test/example27     spin-polarised, fixed occupations

(test/example10-12 add two k-points of zero weight, whose divergence
corrections take the kVaux sums of BAND-mode runs; those are outside this
library's scope, so they are not replayed.)

  qe_si.npz, qe_si_lsda.npz, qe_si_gamma.npz, qe_si_gamma_lsda.npz
                   the QE data TC++ reads (tc_b200.qe.QEData.save_npz, with atoms)
  si_upf.npz       the arrays TC++ reads from Si_test.upf (tc_b200.upf.UPF;
                   every example uses the same file)
  si_examples.json per example: calc_method, its QE fixture, smearing mode and
                   width (input.in), the RPA F of parameters.casl, and the
                   energies TC++ printed after SCF iterations 1 and 2
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

QE_SETS = {"qe_si.npz": "example1", "qe_si_lsda.npz": "example17", "qe_si_gamma.npz": "example26",
           "qe_si_gamma_lsda.npz": "example27"}
EXAMPLES = {"example1": "qe_si.npz", "example2": "qe_si.npz", "example3": "qe_si.npz",
            "example17": "qe_si_lsda.npz", "example18": "qe_si_lsda.npz", "example19": "qe_si_lsda.npz",
            "example26": "qe_si_gamma.npz", "example27": "qe_si_gamma_lsda.npz"}


def parse_input(path):
    """calc_method, smearing mode and width (TC++ defaults: fixed, 0.01 Ha)."""
    opts = {}
    for line in open(path):
        w = line.split()
        if len(w) >= 2:
            opts[w[0]] = w[1]
    return opts["calc_method"], opts.get("smearing_mode", "fixed"), float(opts.get("smearing_width", 0.01))


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
    for fname, ex in QE_SETS.items():
        QEData(os.path.join(test_dir, ex)).save_npz(os.path.join(HERE, fname))
    upf = read_upf(os.path.join(test_dir, "example1", "Si_test.upf"))
    np.savez_compressed(os.path.join(HERE, "si_upf.npz"), **upf.arrays())
    out = {}
    for ex, qe in EXAMPLES.items():
        d = os.path.join(test_dir, ex)
        method, smearing, width = parse_input(os.path.join(d, "input.in"))
        rec = {"calc_method": method, "qe": qe, "smearing": smearing, "smearing_width": width,
               "iterations": parse_output(os.path.join(d, "output.out"))}
        casl = os.path.join(d, "parameters.casl")
        if os.path.exists(casl):
            nspin = 2 if "lsda" in qe else 1
            rec["F"] = read_casl_rpa(casl, nspin=nspin)[1].tolist()
        out[ex] = rec
    with open(os.path.join(HERE, "si_examples.json"), "w") as f:
        json.dump(out, f, indent=1)
    for ex, rec in out.items():
        print(ex, rec["calc_method"], rec.get("F"), rec["iterations"][0].get("2-body"))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/test")
