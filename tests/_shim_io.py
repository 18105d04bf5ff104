"""Binary dump of a TCSystem for tc_b200/shim/shim_check.cpp, build of that
driver, and reading of its results (test infrastructure)."""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "tc_b200", "shim")


def build_driver(out_dir):
    exe = os.path.join(out_dir, "shim_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-DTCG_SHIM_STANDALONE", "-I", SHIM, "-o", exe,
                    os.path.join(SHIM, "shim_check.cpp"), os.path.join(SHIM, "calc_hamiltonian_tcg.cpp"),
                    "-L", os.path.join(ROOT, "tc_b200"), "-ltcg_b200",
                    "-Wl,-rpath," + os.path.join(ROOT, "tc_b200")], check=True)
    return exe


def write_system(s, path, precision=0, owned=None):
    i32 = lambda *v: np.asarray(v, dtype=np.int32).tobytes()
    f64 = lambda v: np.ascontiguousarray(v, dtype=np.float64).tobytes()
    c128 = lambda v: np.ascontiguousarray(v, dtype=np.complex128).tobytes()
    meth = {"HF": 0, "TC": 1, "BITC": 2}[s.method]
    out = [i32(0x53474354, meth, s.nspin, s.nk_irr), i32(*s.nr), i32(s.num_kpoints, len(s.rotation), precision),
           f64(s.lattice), f64(s.recip), f64([s.omega]), i32(*s.nsym_k)]
    for a in range(s.nk_all):
        out += [f64(s.kvec[a]), i32(int(s.rot_index[a]), int(s.time_rev[a]))]
    out.append(i32(*s.npw))
    for sp in range(s.nspin):
        for a in range(s.nk_all):
            gi, ph = s.gidx(sp, a)
            out += [i32(*gi), c128(ph)]
    out += [i32(*np.asarray(s.rotation).ravel()), f64(np.asarray(s.translation).ravel()),
            f64(np.asarray(s.jastrow_A).ravel()), f64(np.asarray(s.jastrow_F).ravel()),
            i32(int(bool(s.includes_div_correction))), f64([s.alpha_Vaux]), f64(s.sum_Vaux),
            i32(*s.nbands), i32(*np.asarray(s.nocc).ravel()), f64(s.filling), c128(s.phik)]
    if s.method == "BITC":
        out.append(c128(s.phik_left))
    out += [c128(s.density), i32(*np.asarray(s.nb_apply).ravel()), c128(s.psi)]
    nbt = int(np.sum(s.nb_apply))
    own = np.ones(nbt, dtype=np.int32) if owned is None else np.asarray(owned, dtype=np.int32)
    out.append(own.tobytes())
    with open(path, "wb") as f:
        f.write(b"".join(out))


def read_result(s, path):
    n = s.psi.size
    raw = open(path, "rb").read()
    c = np.frombuffer(raw[:4 * n * 16], dtype=np.complex128)
    launches = int(np.frombuffer(raw[4 * n * 16:], dtype=np.int64)[0])
    return c[:n], c[n:2 * n], c[2 * n:3 * n], c[3 * n:], launches
