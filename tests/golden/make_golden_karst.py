"""Generates the coupled-model fixtures under tests/golden/ by running the
REFERENCE's own sources (karst.c, reservoir.c, set_source_term.c,
permeabilities.c, solve_linearsystem_AMG.c, flux_reconstruction.c and the
toolbox, compiled from the hmfem tree into oracle/_ref/libhmfem_ref.so by
oracle/Makefile) on the seeded cases of tests/karst_cases.py.

    python tests/golden/make_golden_karst.py

For each case: one conduit() call on a seeded state (keff, source terms,
conduit pressures through compute(), updated fracture velocities) and the
whole coupled run of main.c:383-593 (reservoir and conduit pressures,
conduit fluxes, balances, Picard iterations; the reservoir fluxes as a
digest).  It also copies
two of the reference's conduit data files (data_1_2.dat: the one conduit
of the reference's own run script; data_3_2.dat: three conduits) so the
reader can be checked where the hmfem tree is absent.
"""
import hashlib
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.oracle import Port, Ref  # noqa: E402
import karst_cases as KC  # noqa: E402

REF_TREE = "/root/reference"
DATA_FILES = ("data_1_2.dat", "data_3_2.dat")
STEP_SEED = 5


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    R = Ref()
    P = Port()
    for name, mk in KC.CASES.items():
        prob, k, WI, pw = mk()
        perm, _, _ = P.assemble(prob)
        p_old, pc_old, ucR, ucL = KC.step_state(prob, k, STEP_SEED)
        st = R.conduit_step(k, prob, perm, p_old, pc_old, ucR, ucL, rho=KC.RHO)
        run = R.picard(k, prob, WI, pw, rho=KC.RHO)
        out = dict(K_digest=digest(prob.KX), state_digest=digest(p_old, pc_old, ucR, ucL),
                   perm_digest=digest(perm))
        for key in ("kl", "kr", "kc", "f", "pc", "ucR", "ucL"):
            out["step_" + key] = st[key]
        for key in ("p", "pc", "ucl", "ucr", "qk", "out"):
            out["run_" + key] = run[key]
        out["run_v_digest"] = digest(run["v"])
        out["run_iterations"] = run["iterations"]
        np.savez_compressed(os.path.join(HERE, f"karst_{name}.npz"), **out)
        print(name, "iterations", run["iterations"], "error", run["out"][0])
    for f in DATA_FILES:
        shutil.copyfile(os.path.join(REF_TREE, f), os.path.join(HERE, "karst_" + f))


if __name__ == "__main__":
    main()
