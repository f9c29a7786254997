"""Symmetric 3x3 eigen-decomposition by the cyclic Jacobi method (oracle).

The reference calls Warp's ``wp.eig3`` (mpm/mpm_utils.py:525, 708), whose
algorithm lives in the third-party warp-lang 1.7.0 package and is not
restated here.  The oracle uses the classical cyclic Jacobi eigenvalue
algorithm (Jacobi 1846; Golub & Van Loan, Matrix Computations, section 8.5)
in a form that stays analytic in the matrix entries, so complex-step
derivatives of eigen-dependent quantities come out exact.  Everything built
on it (Hencky/J2/DP/NorSand stresses) is an isotropic function of b, so the
eigenvalue order and eigenvector signs do not matter.
"""
import numpy as np

_PAIRS = ((0, 1), (0, 2), (1, 2))


def eigh3(A, sweeps=8):
    """Batched symmetric eigen-decomposition.

    A: [N, 3, 3] (real or complex).  Returns (lam[N, 3], V[N, 3, 3]) with
    A = V diag(lam) V^T, eigenvectors in the columns of V.
    """
    A = np.array(A, copy=True)
    N = A.shape[0]
    V = np.zeros_like(A)
    V[:, 0, 0] = V[:, 1, 1] = V[:, 2, 2] = 1.0
    for _ in range(sweeps):
        for p, q in _PAIRS:
            apq = A[:, p, q]
            diff = A[:, p, p] - A[:, q, q]
            nz = (np.real(apq) != 0) | (np.imag(apq) != 0)
            dre = np.real(diff)
            with np.errstate(divide="ignore", invalid="ignore"):
                # tan(2 theta) = -2 a_pq / (a_pp - a_qq); principal branch.
                th_reg = -0.5 * np.arctan(2.0 * apq / np.where(dre != 0, diff, 1.0))
            th_deg = np.where(np.real(apq) > 0, -np.pi / 4, np.pi / 4)
            th = np.where(dre != 0, th_reg, th_deg)
            th = np.where(nz, th, 0.0)
            c = np.cos(th)
            s = np.sin(th)
            # G: identity except G[p,p]=c, G[p,q]=s, G[q,p]=-s, G[q,q]=c.
            G = np.zeros_like(A)
            G[:, 0, 0] = G[:, 1, 1] = G[:, 2, 2] = 1.0
            G[:, p, p] = c
            G[:, q, q] = c
            G[:, p, q] = s
            G[:, q, p] = -s
            A = np.einsum("nji,njk,nkl->nil", G, A, G)
            A[:, p, q] = 0.0
            A[:, q, p] = 0.0
            V = np.einsum("nij,njk->nik", V, G)
    lam = np.stack([A[:, 0, 0], A[:, 1, 1], A[:, 2, 2]], 1)
    return lam, V


def from_principal(vals, V):
    """sum_A vals[:, A] n_A n_A^T with n_A = V[:, :, A]."""
    return np.einsum("nia,na,nja->nij", V, vals, V)
