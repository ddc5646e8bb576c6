"""The scalar recurrences of the fused cycle's delayed reorthogonalisation
(arnoldi_fused.cu, DEL = true), restated in numpy with the kernel's
representation (unnormalised basis U with scales sc, pending vector v, the
unrotated Hessenberg matrix), against Arnoldi with classical Gram-Schmidt
and reorthogonalisation: the same Hessenberg matrix, the same orthonormal
basis, and the Arnoldi relation A Q = Q H."""
import numpy as np


def arnoldi_cgs2(A, b, m):
    n = len(b)
    Q = np.zeros((n, m + 1))
    H = np.zeros((m + 1, m))
    Q[:, 0] = b / np.linalg.norm(b)
    for j in range(m):
        w = A @ Q[:, j]
        s = Q[:, :j + 1].T @ w
        w = w - Q[:, :j + 1] @ s
        t = Q[:, :j + 1].T @ w
        w = w - Q[:, :j + 1] @ t
        H[:j + 1, j] = s + t
        H[j + 1, j] = np.linalg.norm(w)
        Q[:, j + 1] = w / H[j + 1, j]
    return Q, H


def arnoldi_delayed(A, b, m):
    """step k: z = A v_k (v_0 = q_0); one reduction of t = U^T v, p = U^T z,
    v.v, v.z; beta, column k-1 of H, the first projection of A q_k from the
    Arnoldi relation; one combine pass writing U_k and v_{k+1}"""
    n = len(b)
    U = np.zeros((n, m + 1))
    sc = np.zeros(m + 2)
    H = np.zeros((m + 1, m))
    U[:, 0] = b
    sc[0] = 1.0 / np.linalg.norm(b)
    v = np.zeros(n)
    hp = np.zeros(m + 2)
    for k in range(m + 1):
        z = A @ (U[:, 0] * sc[0] if k == 0 else v)
        nb = 1 if k == 0 else k
        red = np.concatenate([U[:, :nb].T @ v, U[:, :nb].T @ z, [v @ v, v @ z]])
        if k == 0:
            p0 = sc[0] * red[1]
            hp[0] = p0
            c1, c2, beta, ck = np.zeros(1), np.array([sc[0] * p0]), 1.0, 0.0
        else:
            t = sc[:k] * red[:k]
            p = sc[:k] * red[k:2 * k]
            beta = np.sqrt(red[2 * k] - t @ t)
            H[:k, k - 1] = hp[:k] + t
            H[k, k - 1] = beta
            Ht = H[:k + 1, :k] @ t
            rb = 1.0 / beta
            sk = (red[2 * k + 1] - t @ p - beta * Ht[k]) * rb * rb
            ck = Ht[k] * rb + sk
            si = (p - Ht[:k]) * rb
            c1 = sc[:k] * t
            c2 = sc[:k] * (Ht[:k] * rb + si - ck * t * rb)
            hp[:k], hp[k], sc[k] = si, sk, rb
            if k == m:
                break
        rb = 1.0 if k == 0 else 1.0 / beta
        vcoef = 0.0 if k == 0 else ck * rb
        acc1, acc2 = U[:, :nb] @ c1, U[:, :nb] @ c2
        if k >= 1:
            U[:, k] = v - acc1
        v = z * rb - vcoef * v - acc2
    return U[:, :m] * sc[:m], H


def test_delayed_recurrences_match_cgs2_arnoldi():
    rng = np.random.default_rng(0)
    n, m = 200, 30
    A = np.eye(n) * 4 + rng.standard_normal((n, n)) * 0.3
    b = rng.standard_normal(n)
    Q1, H1 = arnoldi_cgs2(A, b, m)
    Q2, H2 = arnoldi_delayed(A, b, m)
    assert np.abs(H1 - H2).max() < 1e-12
    assert np.abs(Q1[:, :m] - Q2).max() < 1e-12
    assert np.abs(Q2.T @ Q2 - np.eye(m)).max() < 1e-12
    # A Q_{m-1} = Q_m H_{0..m-1, 0..m-2}
    assert np.abs(A @ Q2[:, :m - 1] - Q2 @ H2[:m, :m - 1]).max() < 1e-12
