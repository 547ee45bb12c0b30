"""Oracle (test infrastructure only): CPU restatement of TigerCI's standard
Davidson-Liu solver, tiger_fortran/davidson.f90:47-239, with
  expand_krylov_subspace ... :478-494
  build_residual_std_eig ... :503-526
  is_converged ............. :564-602
  build_next_vector_std_eig  :609-631  (r <- -r/(H_ii - E), 0 when equal)
  build_wavefunction ....... :675-694
  orthonormalize_vector .... :702-723  (MGS, renormalised after every projection)
  init_from_diag ........... initial_davidson_guess.f90:99-137
  need_to_restart_subspace / restart_davidson_subspace
  ........................... davidson_restart.f90:26-139 (when disk_space is
                              given: more than 4 vectors per root and
                              2 * num_vec * n * 8 bytes >= disk_space)
and numpy's symmetric eigensolver in place of dsyev.  Vectors are kept in
memory instead of on disk.  A restart keeps the current and the previous
Ritz vector of every unconverged root (the current one of a converged root);
the reference orthonormalises each root's pair on its own, which for one root
is the same thing; for several roots this restatement orthonormalises the
whole collapsed set, so that the basis stays orthonormal.
"""
from __future__ import annotations

import numpy as np


def davidson_liu(sigma, hdiag, roots=1, tol_residual=1e-6, tol_energy=1e-6, maxit=None, disk_space=None):
    n = len(hdiag)
    maxit = maxit or 50 * roots
    order = np.lexsort((np.arange(n), hdiag))[:roots]
    C = [np.zeros(n) for _ in range(roots)]
    for k in range(roots):
        C[k][order[k]] = 1.0
    HC = [None] * roots
    hsub = np.zeros((0, 0))
    energy = np.zeros(roots)
    root2index = list(range(roots))
    converged = [False] * roots
    restarted = set()
    V = None
    it = 0
    for it in range(1, maxit + 1):
        for q in range(roots):
            if converged[q]:
                continue
            idx = root2index[q]
            s = sigma(C[idx])
            while len(HC) <= idx:
                HC.append(None)
            HC[idx] = s
            m = idx + 1
            if hsub.shape[0] < m:
                h2 = np.zeros((m, m))
                h2[:hsub.shape[0], :hsub.shape[0]] = hsub
                hsub = h2
            for k in range(m):
                hsub[k, idx] = hsub[idx, k] = C[k] @ s
        num_vec = len(C)
        prevV = V
        w, V = np.linalg.eigh(hsub[:num_vec, :num_vec])
        dE = np.abs(w[:roots] - energy)
        energy = w[:roots].copy()
        if disk_space is not None and num_vec > 4 * roots and 16.0 * n * num_vec >= disk_space:
            restarted.add(it)
            B = [V[:, q].copy() for q in range(roots)]
            if prevV is not None:
                for q in range(roots):
                    if not converged[q]:
                        b = np.zeros(num_vec)
                        b[:prevV.shape[0]] = prevV[:, q]
                        B.append(b)
            Q = []
            for b in B:
                for qv in Q:
                    b = b - (qv @ b) * qv
                nb = np.linalg.norm(b)
                if nb >= 1e-8 and len(Q) < 2 * roots:
                    Q.append(b / nb)
            Q = np.array(Q).T  # num_vec x m
            C = [sum(Q[k, j] * C[k] for k in range(num_vec)) for j in range(Q.shape[1])]
            HC = [sum(Q[k, j] * HC[k] for k in range(num_vec)) for j in range(Q.shape[1])]
            hsub = Q.T @ hsub[:num_vec, :num_vec] @ Q
            hsub = 0.5 * (hsub + hsub.T)
            num_vec = len(C)
            w, V = np.linalg.eigh(hsub)
            energy = w[:roots].copy()
        for q in range(roots):
            if converged[q]:
                continue
            a = V[:, q]
            r = sum(a[k] * (HC[k] - energy[q] * C[k]) for k in range(num_vec))
            norm = np.sqrt(r @ r)
            if it not in restarted and (it - 1) not in restarted and (
                    norm < tol_residual or (abs(dE[q]) < tol_energy and it > 1) or it == maxit):
                converged[q] = True
                continue
            p = hdiag - energy[q]
            r = np.where(p == 0.0, 0.0, -r / np.where(p == 0.0, 1.0, p))
            for k in range(len(C)):
                r = r - (r @ C[k]) * C[k]
                nr = np.sqrt(r @ r)
                r = np.zeros(n) if abs(nr) < 1e-14 else r / nr
            C.append(r)
            root2index[q] = len(C) - 1
        if all(converged):
            break
    num_vec = len(C)
    w, V = np.linalg.eigh(hsub[:num_vec, :num_vec])
    vecs = []
    for q in range(roots):
        v = sum(V[k, q] * C[k] for k in range(num_vec))
        vecs.append(v / np.linalg.norm(v))
    return energy, np.array(vecs), min(it, maxit)
