"""Generate the committed regression fixtures tests/golden/*.npz.

Each fixture holds the oracle's H2 psi / H3 psi for a small seeded system
(tc_b200.synth.small), so the oracle (CPU tests) and the CUDA library (GPU
tests) are checked against frozen numbers.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tc_b200 import abi, synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    "small_hf": dict(method="HF", nr=(12, 12, 12), nk=2, ecut=2.5, nbands=3, nocc=2, seed=11),
    "small_tc": dict(method="TC", nr=(12, 12, 12), nk=2, ecut=2.5, nbands=3, nocc=2, seed=12),
    "small_bitc": dict(method="BITC", nr=(12, 12, 12), nk=2, ecut=2.5, nbands=3, nocc=2, seed=13),
    "small_bitc_tr": dict(method="BITC", nr=(16, 16, 16), ecut=1.5, nbands=2, nocc=1, seed=14, tr=True),
}


def system(name):
    return synth.small(**CASES[name])


def mask_of(s):
    return abi.TERMS_HF if s.method == "HF" else abi.TERMS_TC


def main():
    for name in CASES:
        s = system(name)
        h2, h3 = O.apply(s, mask_of(s))
        per = {}
        for t, bit in abi.TERM_NAMES.items():
            if bit & mask_of(s):
                a, b = O.apply(s, bit)
                per[t] = a if bit & abi.TERMS_H2 else b
        np.savez_compressed(os.path.join(HERE, name + ".npz"), h2=h2, h3=h3, psi=s.psi,
                            **{"term_" + k: v for k, v in per.items()})
        print(name, s.method, "npw", list(s.npw), "|h2|", float(np.abs(h2).max()), "|h3|", float(np.abs(h3).max()))


if __name__ == "__main__":
    main()
