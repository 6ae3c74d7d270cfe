"""Generates the golden fixtures under tests/golden/ by running the
REFERENCE's own sources (oracle/_ref/libhmfem_ref.so, compiled from the hmfem
tree by oracle/Makefile) on seeded synthetic problems.

    python tests/golden/make_golden.py

Small cases store every array; larger cases store SHA-256 digests of every
array (inputs, matrix, each hierarchy level's structure and values, one
V-cycle, the PCG iterates at the reference's stopping rule and at 1e-12,
the fluxes), which the oracle must reproduce bit for bit.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Ref  # noqa: E402
from hmfem_b200.problem import config_problem, make_problem  # noqa: E402

CASES = {
    # small, mixed boundary types, heterogeneous K with conduits
    "mixed_7x5x6": lambda: make_problem(
        7, 5, 6, log10k=(-14.0, 1.0, 1.5), n_conduits=2, seed=3,
        bc_type=(0, 1, 0, 1, 0, 1), bc_value=(2.0, 0.5, 1.0, -0.3, 0.0, 0.7)),
    "allneumann_6x4x5": lambda: make_problem(
        6, 4, 5, log10k=(-13.0, 0.5, 1.0), seed=5, bc_type=(1,) * 6,
        bc_value=(0.1, 0.1, 0.0, 0.0, 0.0, 0.0)),
    "config0_32": lambda: config_problem(0),
    "config1_24": lambda: config_problem(1, size=24),
    "config2_20": lambda: config_problem(2, size=20),
}
FULL = {"mixed_7x5x6", "allneumann_6x4x5"}


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    R = Ref()
    for name, mk in CASES.items():
        p = mk()
        perm, ind, b = R.assemble(p)
        cnt, col, ele = R.pack(p, perm, ind)
        H = R.hierarchy(cnt, col, ele)
        f = np.random.default_rng(7).standard_normal(p.n)
        uf = R.vcycle(f)
        x8, it8, rel8, _, _ = R.compute(cnt, col, ele, b, eps=1e-8, stop=1)
        x, it, rel, _, _ = R.compute(cnt, col, ele, b, eps=1e-12, stop=2)
        v = R.fluxes(p, perm, x)
        faces6 = v[:, [0, 1, 2, 3, 5, 6]]
        out = dict(nx=p.nx, ny=p.ny, nz=p.nz, hx=p.hx, hy=p.hy, hz=p.hz,
                   bc_type=np.array(p.bc_type), bc_value=np.array(p.bc_value),
                   iters_ref8=it8, iters=it, relres=rel,
                   K_digest=digest(p.KX), b_digest=digest(b),
                   vcycle_digest=digest(uf), x_ref8_digest=digest(x8),
                   x_digest=digest(x), flux_digest=digest(faces6),
                   x_sample=x[:: max(1, p.n // 16)],
                   nlevels=len(H.levels),
                   level_n=np.array([d["n"] for d in H.levels]),
                   level_nnz=np.array([len(d["col"]) for d in H.levels]),
                   level_pnnz=np.array([len(d["pcol"]) for d in H.levels]),
                   csr_digest=digest(cnt, col, ele))
        for l, d in enumerate(H.levels):
            out[f"L{l}_struct"] = digest(d["cnt"], d["col"], d["sel"], d["pcnt"],
                                         d["pcol"])
            out[f"L{l}_values"] = digest(d["ele"], d["dinv"], d["pele"])
            if name in FULL:
                for k, a in d.items():
                    if k != "n":
                        out[f"L{l}_{k}"] = a
        if name in FULL:
            out.update(perm=perm, ind=ind, cnt=cnt, col=col, ele=ele, K=p.KX,
                       b=b, vcycle_u=uf, x_ref8=x8, x=x, flux=faces6)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, p.n, "levels", len(H.levels), "iters", it8, it, "relres", rel)


if __name__ == "__main__":
    main()
