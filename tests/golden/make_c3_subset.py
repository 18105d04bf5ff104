"""Generate tests/golden/c3_subset.npz: the oracle's H2 psi / H3 psi of a
subset of bands of the C3 workload, and the oracle's FP64 energy terms of its
occupied orbitals.

C3 = batched BITC apply (fcc Si, 4x4x4 mesh, 14 Ha, 36^3, 16 bands per k, 4
occupied, left / right orbitals from seeds 1 / 2; tc_b200.synth.config).  The
full apply is 1024 band-applies, far beyond what the CPU oracle finishes in a
test, so the fixture holds
  - SUBSET: the oracle's H2 psi and H3 psi of a dozen (k, band) targets
    spread over the mesh (occupied and trial bands), all terms, every
    occupied source in the q-sums;
  - E2, E3: the oracle's two- and three-body energies (total_energy.cpp:101-168,
    e_n = <chi_i|H_n phi_i>) from H applied to all occupied orbitals.
The GPU tests and bench.py compare the CUDA path (FP64 and mixed precision)
against these numbers.  Run from the repository root (on
eight cores, about an hour):

    python tests/golden/make_c3_subset.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tc_b200 import abi, synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

# (k, band) targets of the parity subset: occupied (band < 4) and trial bands
SUBSET = [(0, 0), (0, 15), (9, 3), (9, 4), (21, 1), (27, 8), (36, 2), (42, 11), (50, 5), (55, 3), (60, 0), (63, 14)]


def owned_mask(s, pairs):
    nb = int(s.nb_apply[0][0])
    m = np.zeros(s.nspin * s.nk_irr * nb, dtype=np.uint8)
    for k, b in pairs:
        m[k * nb + b] = 1
    return m


def occupied_pairs(s):
    return [(k, b) for k in range(s.nk_irr) for b in range(int(s.nocc[0][k]))]


def main():
    t0 = time.time()
    s = synth.config("C3")
    print("built C3", round(time.time() - t0, 1), "s", flush=True)
    pairs = sorted(set(SUBSET) | set(occupied_pairs(s)))
    owned = owned_mask(s, pairs)
    h2, h3 = O.apply(s, abi.TERMS_TC, owned=owned)
    print("oracle apply", round(time.time() - t0, 1), "s", flush=True)
    e2, e3 = s.energy_terms(h2, h3)
    sub2 = [s.band_view(h2, 0, k, b) for k, b in SUBSET]
    sub3 = [s.band_view(h3, 0, k, b) for k, b in SUBSET]
    np.savez_compressed(os.path.join(HERE, "c3_subset.npz"), subset=np.array(SUBSET, dtype=np.int32),
                        h2=np.concatenate(sub2), h3=np.concatenate(sub3), E2=np.complex128(e2),
                        E3=np.complex128(e3))
    print("E2", e2, "E3", e3, "total", round(time.time() - t0, 1), "s")


if __name__ == "__main__":
    main()
