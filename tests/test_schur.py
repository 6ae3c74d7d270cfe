"""The exact red-black reduction (hmfem_options.schur0): its level-1
restatement (oracle/schur.py) against the algebra it stands for, on CPU."""
import numpy as np
import scipy.sparse as sp

from hmfem_b200.problem import make_problem
from oracle import schur as S


def _csr(cnt, col, ele):
    ptr = np.zeros(len(cnt) + 1, np.int64)
    ptr[1:] = np.cumsum(cnt)
    return sp.csr_matrix((ele, col, ptr), shape=(len(cnt), len(cnt)))


def test_restatement_is_the_schur_complement(port):
    p = make_problem(7, 6, 5, log10k=(-14.0, 1.0, 1.5), n_conduits=1, seed=4,
                     bc_type=(0, 1, 0, 1, 0, 1), bc_value=(1.0, 0.5, 0.0, 0.0, 0.2, 0.0))
    perm, ind, b = port.assemble(p)
    cnt, col, ele = port.pack(perm, ind)
    A = _csr(cnt, col, ele)
    S1 = _csr(*S.schur_level1(perm, p.nx, p.ny, p.nz))
    G = S.galerkin_direct(A, p.nx, p.ny, p.nz)
    assert S1.shape == G.shape
    D = (S1 - G).tocoo()
    assert np.abs(D.data).max() <= 1e-13 * np.abs(G.data).max()
    # same rows and columns as the reference's level 1 (P^T A P with the
    # averaging interpolation)
    H = port.amg(cnt, col, ele)
    L1 = H.level(1)
    assert np.array_equal(L1["cnt"], np.diff(S1.indptr).astype(np.int32))
    assert np.array_equal(L1["col"], S1.indices.astype(np.int32))
    # symmetric, positive diagonal, non-positive couplings (an M-matrix)
    assert abs(S1 - S1.T).max() <= 1e-15 * abs(S1).max()
    off = S1 - sp.diags(S1.diagonal())
    assert off.max() <= 0 and S1.diagonal().min() > 0
