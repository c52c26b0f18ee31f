"""Test helper: a numpy restatement of the library's s-step (block) GMRES with orthonormalised block storage.

It follows the algebra of ``gmres_block`` in the CUDA library, written here with an explicit orthonormal basis:
s classical Gram-Schmidt steps whose Ritz values (Leja-ordered) are the first Newton shifts, then blocks of s operator
applications Y_t = (M^-1 A - theta_t) Y_{t-1} from Y_0 = V_m (each block's shifts are the Ritz values of the
previous block's diagonal Hessenberg block), one block Gram-Schmidt projection, a Cholesky QR of
the projected block, and the Hessenberg columns recovered from (M^-1 A) V W_{0:s-1} = V (W_{1:s} + W_{0:s-1} theta).
Givens rotations and the stopping test run column by column, as in ``oracle.cbs_oracle.gmres`` (Krylov.jl
semantics), so in exact arithmetic the iterate is that of full GMRES.
"""
from __future__ import annotations

import numpy as np

from oracle import cbs_oracle as O


def leja(values):
    """Leja ordering: largest modulus first, then each next value maximises the product of distances."""
    vals = list(values)
    if not vals:
        return vals
    out = [max(vals, key=abs)]
    vals.remove(out[0])
    while vals:
        nxt = max(vals, key=lambda z: np.prod([abs(z - w) for w in out]))
        out.append(nxt)
        vals.remove(nxt)
    return out


def block_gmres(apply_A, apply_M, b, x0, atol, rtol, itmax, s):
    shape = b.shape
    if b.ndim != 1:  # fields: work on flat vectors, return the field shape
        fA, fM = apply_A, apply_M
        res = block_gmres(lambda v: fA(v.reshape(shape)).ravel(), lambda v: fM(v.reshape(shape)).ravel(),
                          b.ravel(), x0.ravel(), atol, rtol, itmax, s)
        res.x = res.x.reshape(shape)
        return res
    x = x0.copy()
    r0 = apply_M(b - apply_A(x))
    beta = O._nrm(r0)
    if beta == 0:
        return O.KrylovResult(x, 0, True, [beta])
    eps = atol + rtol * beta
    btol = np.finfo(np.float64).eps ** 0.75
    V = [r0 / beta]
    Hc = []            # Hessenberg columns (length m + 2 each)
    R = []             # rotated columns
    cs, ss = [], []
    z = [complex(beta)]
    rn = [beta]
    state = {"solved": beta <= eps, "done": False}

    def rotate(col):
        """Apply the previous rotations and a new one to Hessenberg column j = len(R); True when the solve stops.
        The subdiagonal entry is real: |w| in the Gram-Schmidt steps, Rb[c, c] / T[c, c] in a block."""
        j = len(R)
        hb = float(np.real(col[j + 1]))
        col = list(col[: j + 1])
        for i in range(j):
            t = cs[i] * col[i] + ss[i] * col[i + 1]
            col[i + 1] = np.conj(ss[i]) * col[i] - cs[i] * col[i + 1]
            col[i] = t
        c, sn, rho = O.sym_givens(col[j], hb)
        col[j] = rho
        cs.append(c)
        ss.append(sn)
        R.append(col[: j + 1])
        zk1 = np.conj(sn) * z[j]
        z[j] = c * z[j]
        z.append(zk1)
        rn.append(abs(zk1))
        state["solved"] = abs(zk1) <= eps or abs(zk1) + 1.0 <= 1.0
        return state["solved"] or hb <= btol or len(R) >= itmax

    # phase 1: s classical Gram-Schmidt steps
    m = 0
    while not state["done"] and m < s and not state["solved"]:
        w = apply_M(apply_A(V[m]))
        h = [O._dot(v, w) for v in V]
        for hi, v in zip(h, V):
            w = w - hi * v
        hb = O._nrm(w)
        col = h + [complex(hb)]
        Hc.append(col)
        state["done"] = rotate(col)
        if not state["done"]:
            V.append(w / hb)
        m += 1
    theta = [0j] * s
    if not state["done"] and m == s:
        Hs = np.array([[Hc[j][i] if i < len(Hc[j]) else 0 for j in range(s)] for i in range(s)])
        theta = leja(list(np.linalg.eigvals(Hs)))

    # phase 2: blocks
    while not state["done"] and len(R) < itmax:
        K = m + 1
        Y = [V[m]]
        for t in range(1, s + 1):
            Y.append(apply_M(apply_A(Y[-1])) - theta[t - 1] * Y[-1])
        Vm = np.stack(V[:K], axis=1)
        Yb = np.stack(Y[1:], axis=1)
        D = Vm.conj().T @ Yb
        Yp = Yb - Vm @ D
        G = Yp.conj().T @ Yp
        try:
            L = np.linalg.cholesky(G)        # G = L L^H, Rb = L^H
        except np.linalg.LinAlgError:
            break
        Rb = L.conj().T
        Vn = Yp @ np.linalg.inv(Rb)
        n = K + s
        W = np.zeros((n, s + 1), dtype=complex)
        W[m, 0] = 1.0
        W[:K, 1:] = D
        W[K:, 1:] = Rb
        Rh = W[:, 1:] + W[:, :s] * np.array(theta)[None, :]
        Hold = np.zeros((n, m), dtype=complex)
        for j in range(m):
            Hold[: len(Hc[j]), j] = Hc[j]
        Rh = Rh - Hold @ W[:m, :s]
        T = W[m:m + s, :s]
        Hn = Rh @ np.linalg.inv(T)
        V.extend(Vn[:, c] for c in range(s))
        for c in range(s):
            col = list(Hn[: m + c + 2, c])
            Hc.append(col)
            if rotate(col):
                state["done"] = True
                break
        m += s
        if not state["done"]:  # next shifts: Ritz values of this block's s x s diagonal Hessenberg block
            Hs = np.array([[Hc[m - s + j][m - s + i] if m - s + i < len(Hc[m - s + j]) else 0 for j in range(s)]
                           for i in range(s)])
            theta = leja(list(np.linalg.eigvals(Hs)))

    k = len(R)
    y = list(z[:k])
    for i in range(k - 1, -1, -1):
        for j in range(k - 1, i, -1):
            y[i] = y[i] - R[j][i] * y[j]
        if abs(R[i][i]) <= btol:
            y[: i + 1] = [0j] * (i + 1)
            break
        y[i] = y[i] / R[i][i]
    for i in range(k):
        x = x + y[i] * V[i]
    return O.KrylovResult(x, k, bool(state["solved"]), rn)
