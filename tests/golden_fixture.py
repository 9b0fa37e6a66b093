"""Loads a golden fixture (tests/golden/*.npz, written by tests/golden/make_golden.py from the
reference's own outputs) into a Setup with the reference's exact partition, ghost lists, partition
of unity, coarse basis and local factors, plus the reference's outputs to compare against."""
from __future__ import annotations

import os

import numpy as np
import scipy.sparse as sp

from s2l_b200.setup_phase import LocalFactor, SchwarzOptions, Setup, SubdomainData, coarse_matrix

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KINDS = {0: "lu", 1: "llt", 2: "ldlt"}


def cases():
    # the AMG fixtures (amg_*.npz) and the generator fixture (*_generator.npz) are of other kinds
    return sorted(f[:-4] for f in os.listdir(GOLDEN)
                  if f.endswith(".npz") and not f.startswith("amg_") and not f.endswith("_generator.npz"))


def _flag(cmd: list, name: str, default: str) -> str:
    """Value of the last occurrence of a flag (the reference's parser keeps the last one)."""
    idx = [i for i, a in enumerate(cmd) if a == name]
    return cmd[idx[-1] + 1] if idx else default


def load(name: str):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    cmd = str(d["command"]).split()
    n, nsub, symmetric, n0 = (int(v) for v in d["global_meta"])
    A = sp.csr_matrix((d["global_A_v"], d["global_A_ci"], d["global_A_rp"]), shape=(n, n))
    opts = SchwarzOptions(one_level=_flag(cmd, "--one-level", "ras"), coarse=_flag(cmd, "--coarse", "deflated"),
                          pou=_flag(cmd, "--pou", "boolean"), overlap=1,
                          local_precision=_flag(cmd, "--local-precision", "double"))
    subs = []
    for i in range(nsub):
        p = f"sub{i}_"
        begin, n_owned, n_ghost, m = (int(v) for v in d[p + "meta"])
        nl = n_owned + n_ghost
        kind, single = (int(v) for v in d[p + "fmeta"])
        dt = np.float32 if single else np.float64
        L = sp.csr_matrix((d[p + "L_v"].astype(dt), d[p + "L_ci"], d[p + "L_rp"]), shape=(nl, nl))
        U = (sp.csr_matrix((d[p + "U_v"].astype(dt), d[p + "U_ci"], d[p + "U_rp"]), shape=(nl, nl))
             if kind == 0 else None)
        f = LocalFactor(KINDS[kind], L, U, d[p + "pin"].astype(np.int32), d[p + "pout"].astype(np.int32),
                        d[p + "d"].astype(dt) if kind == 2 else None)
        V = d[p + "V"].reshape(m, nl).T.copy() if (p + "V") in d else np.zeros((nl, 0))
        Aii = sp.csc_matrix((d[p + "Aii_v"], d[p + "Aii_ri"], d[p + "Aii_cp"]), shape=(nl, nl)).tocsr()
        subs.append(SubdomainData(begin, n_owned, d[p + "ghosts"].astype(np.int64), d[p + "D"], f, V, Aii))
    offsets = d["global_coarse_offsets"] if "global_coarse_offsets" in d else np.zeros(nsub + 1, dtype=np.int64)
    st = Setup(A, d["global_b"], d["global_ownership"], subs, offsets.astype(np.int64), np.zeros((0, 0)), opts,
               bool(symmetric), d["global_new_to_old"], name)
    if opts.coarse != "none" and n0 > 0:
        st.E = coarse_matrix(A, subs, st.offsets)
    krylov = {"method": _flag(cmd, "--krylov", "gmres"), "restart": int(_flag(cmd, "--restart", "30")),
              "rtol": float(_flag(cmd, "--rtol", "1e-8")), "x": d["krylov_x"], "history": d["krylov_history"],
              "iterations": int(d["krylov_meta"][0]), "converged": bool(d["krylov_meta"][1]),
              "true_rel_residual": float(d["krylov_meta"][3]),
              "stop_norm": _flag(cmd, "--stop-norm", "l2"), "atol": float(_flag(cmd, "--atol", "0"))}
    if d["krylov_meta"].size >= 8:  # OpenFOAM normalised residuals (include/solver/krylov.hpp:51-52)
        krylov["initial_residual_of"] = float(d["krylov_meta"][6])
        krylov["final_residual_of"] = float(d["krylov_meta"][7])
    applies = []
    k = 0
    while f"apply{k}_r" in d:
        q = f"apply{k}_"
        applies.append({key[len(q):]: d[key] for key in d if key.startswith(q)})
        k += 1
    local = [(d[f"sub{i}_ls_b"], d[f"sub{i}_ls_x"]) for i in range(nsub)]
    return st, applies, krylov, local
