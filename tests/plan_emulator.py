"""numpy replay of a pass plan: applies the expanded gates in the order the
scheduler chose (pass by pass), so the reordering can be checked on the CPU
against the oracle without a GPU."""
import numpy as np

K_G1, K_DIAG, K_SWAP, K_U2 = 0, 1, 2, 3
G1_HF, G1_X, G1_Y, G1_RX, G1_RY, G1_GEN, G1_H = 0, 1, 2, 3, 4, 5, 7


def g1_matrix(sub, m):
    if sub == G1_H:
        f = m[0].real
        return np.array([[f, f], [f, -f]], dtype=np.complex128)
    if sub == G1_X:
        return np.array([[0, 1], [1, 0]], dtype=np.complex128)
    if sub == G1_Y:
        return np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    if sub == G1_RX:
        c, s = m[0].real, m[0].imag
        return np.array([[c, -1j * s], [-1j * s, c]], dtype=np.complex128)
    if sub == G1_RY:
        c, s = m[0].real, m[0].imag
        return np.array([[c, -s], [s, c]], dtype=np.complex128)
    return np.array([[m[0], m[1]], [m[2], m[3]]], dtype=np.complex128)


def replay(n, plan, psi=None):
    N = 1 << n
    if psi is None:
        psi = np.zeros(N, dtype=np.complex128)
        psi[0] = 1.0
    psi = psi.copy()
    idx = np.arange(N, dtype=np.uint64)
    seq = sorted(range(len(plan["pass_of"])), key=lambda i: (plan["pass_of"][i], plan["order"][i]))
    for i in seq:
        kind, sub = divmod(int(plan["kind"][i]), 16)
        t, t2, lo, hi = (int(x) for x in plan["qubits"][i])
        cm = np.uint64(lo | (hi << 32))
        m = plan["matrix"][i]
        cond = (idx & cm) == cm
        if kind == K_G1:
            U = g1_matrix(sub, m)
            b = np.uint64(1 << t)
            i0 = idx[((idx & b) == 0) & cond]
            i1 = i0 | b
            a0, a1 = psi[i0].copy(), psi[i1].copy()
            psi[i0] = U[0, 0] * a0 + U[0, 1] * a1
            psi[i1] = U[1, 0] * a0 + U[1, 1] * a1
        elif kind == K_DIAG:
            if sub & 1:
                psi[cond] = -psi[cond]
            elif t != 0xFFFFFFFF:
                sel = ((idx >> np.uint64(t)) & np.uint64(1)) == 1
                psi[cond & sel] *= m[1]
                psi[cond & ~sel] *= m[0]
            else:
                psi[cond] *= m[0]
        elif kind == K_SWAP:
            b1, b2 = np.uint64(1 << t), np.uint64(1 << t2)
            base = idx[((idx & (b1 | b2)) == 0) & cond]
            x, y = base | b2, base | b1
            psi[x], psi[y] = psi[y].copy(), psi[x].copy()
        elif kind == K_U2:
            bl, bh = np.uint64(1 << t), np.uint64(1 << t2)
            base = idx[(idx & (bl | bh)) == 0]
            grp = [base, base | bl, base | bh, base | bl | bh]
            vals = np.stack([psi[g] for g in grp])
            U = m.reshape(4, 4)
            out = U @ vals
            for r in range(4):
                psi[grp[r]] = out[r]
        else:
            raise AssertionError(f"unexpected kind {kind}")
    return psi / np.linalg.norm(psi)
