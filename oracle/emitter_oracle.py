"""CPU oracle of the EmitterMPS sampler (chi x chi emitter, L labels per photon).

TEST INFRASTRUCTURE.  Only `tests/` and `bench.py`'s CPU-baseline arm may import this module; the product
path (`photonic_engines_b200`) never does.

What it restates (file:line in the reference project):
  coefficient tensor c[x, s_f]                 photonic_engines/clifford/emitter_reference.py:43-51
  reduced density of the placed photons        emitter_reference.py:89-95
  candidate weights by the density method      emitter_reference.py:98-120 (Laplace along the new row)
  the sampler's use of the generator           photonic_engines/clifford/emitter_sampler.py:100-180
  matrix-cofactor weights from given terms     emitter_reference.py:280-305 (matrix_weights)
`candidate_weights` comes from the explicit reduced density matrix and Ryser permanents: an algorithm
independent of the gap-channel decomposition and the matrix-cofactor sums the GPU path uses;
`matrix_weights` restates those sums on the CPU, for steps too large for the density method.
"""
from __future__ import annotations

import itertools
import math

import numpy as np

from .oracle import per_ryser


def coefficient_tensor(ops, s0) -> np.ndarray:
    """c[x_0, ..., x_{n-1}, s] = (M_{n-1, x_{n-1}} ... M_{0, x_0} s0)[s], shape [L]*n + [chi]."""
    ops = np.asarray(ops, dtype=np.complex128)
    n, L, chi, _ = ops.shape
    v = np.asarray(s0, dtype=np.complex128).reshape(1, chi)
    for k in range(n):
        v = np.einsum("lts,bs->blt", ops[k], v).reshape(-1, chi)
    return v.reshape(*([L] * n), chi)


def final_distribution(ops, s0) -> np.ndarray:
    c = coefficient_tensor(ops, s0)
    p = (np.abs(c) ** 2).reshape(-1, c.shape[-1]).sum(0)
    return p


def reduced_density(c_pure: np.ndarray, T) -> np.ndarray:
    """rho_T [L^k, L^k] of the label tensor c_pure [L]*n over the slots T (in the order of T)."""
    n = c_pure.ndim
    rest = [j for j in range(n) if j not in T]
    L = c_pure.shape[0]
    mat = np.transpose(c_pure, list(T) + rest).reshape(L ** len(T), -1)
    return mat @ mat.conj().T


def candidate_weights(U, ops, modes, s0, final, T, rows) -> np.ndarray:
    """w(rho) for every output mode rho, after `rows` for the placed slots T (sorted); `final` the
    projection vector [chi]."""
    U = np.asarray(U, dtype=np.complex128)
    m = U.shape[0]
    c = np.einsum("...s,s->...", coefficient_tensor(ops, s0), np.conj(np.asarray(final, dtype=np.complex128)))
    L = c.shape[0]
    T = list(T)
    k = len(T)
    rho_T = reduced_density(c, T)
    V = np.zeros((m, L ** k), dtype=np.complex128)
    for xi, x in enumerate(itertools.product(range(L), repeat=k)):
        cols = [modes[T[j]][x[j]] for j in range(k)]
        for cc in range(k):
            sub = U[np.ix_(list(rows), [cols[j] for j in range(k) if j != cc])]
            V[:, xi] += U[:, cols[cc]] * per_ryser(sub)
    return np.maximum(np.einsum("rx,xy,ry->r", V, rho_T, V.conj()).real, 0.0)


def exact_distribution(U, ops, modes, s0, final=None) -> dict:
    """{occupation tuple: probability} of the n photons through U: sum over final spins (traced emitter)
    of |sum_x c_x per(U[rows(o), modes(x)])|^2 / prod o!."""
    U = np.asarray(U, dtype=np.complex128)
    m = U.shape[0]
    ops = np.asarray(ops, dtype=np.complex128)
    n, L, chi, _ = ops.shape
    ctens = coefficient_tensor(ops, s0)
    finals = [np.asarray(final, dtype=np.complex128)] if final is not None else list(np.eye(chi))
    xs = list(itertools.product(range(L), repeat=n))
    dist = {}
    for t in itertools.combinations_with_replacement(range(m), n):
        occ = np.bincount(t, minlength=m)
        pers = np.array([per_ryser(U[np.ix_(list(t), [modes[j][x[j]] for j in range(n)])]) for x in xs])
        p = 0.0
        for fv in finals:
            cx = np.array([np.dot(ctens[x], np.conj(fv)) for x in xs])
            p += abs(np.dot(cx, pers)) ** 2
        dist[tuple(int(v) for v in occ)] = p / np.prod([math.factorial(int(v)) for v in occ])
    tot = sum(dist.values())
    return {k_: v / tot for k_, v in dist.items()}


def subset_distribution(U, ops, modes, s0, final, T) -> dict:
    """{occupation: probability} of the photons in slots T with every other photon traced out (lost):
    P(o) = sum_{x, y} rho_T[x, y] per(U[rows(o), modes_T(x)]) conj(per(U[rows(o), modes_T(y)])) / prod o!,
    rho_T the reduced density of the label tensor over T (a traced emitter's spin traced with the rest)."""
    U = np.asarray(U, dtype=np.complex128)
    m = U.shape[0]
    ops = np.asarray(ops, dtype=np.complex128)
    n, L, chi, _ = ops.shape
    c = coefficient_tensor(ops, s0)
    if final is not None:
        c = np.einsum("...s,s->...", c, np.conj(np.asarray(final, dtype=np.complex128)))
    T = list(T)
    k = len(T)
    rho_T = reduced_density(c, T)
    xs = list(itertools.product(range(L), repeat=k))
    dist = {}
    for t in itertools.combinations_with_replacement(range(m), k):
        occ = np.bincount(t, minlength=m)
        pers = np.array([per_ryser(U[np.ix_(list(t), [modes[T[j]][x[j]] for j in range(k)])]) for x in xs])
        p = float(np.einsum("x,xy,y->", pers, rho_T, pers.conj()).real)
        dist[tuple(int(v) for v in occ)] = p / np.prod([math.factorial(int(v)) for v in occ])
    tot = sum(dist.values())
    return {k_: v / tot for k_, v in dist.items()}


def lossy_distribution(U, ops, modes, s0, final, eta: float) -> dict:
    """Law under uniform input-side loss: every photon survives independently with probability eta, the
    lost ones are traced out (the reference's docs/LOSS.md model for emitters)."""
    n = np.asarray(ops).shape[0]
    m = np.asarray(U).shape[0]
    dist: dict = {}
    for r in range(n + 1):
        for T in itertools.combinations(range(n), r):
            w = eta ** r * (1 - eta) ** (n - r)
            part = subset_distribution(U, ops, modes, s0, final, T) if T else {tuple([0] * m): 1.0}
            for k_, p in part.items():
                dist[k_] = dist.get(k_, 0.0) + w * p
    return dist


def sample(U, ops, modes, s0, final, shots: int, generator) -> np.ndarray:
    """Occupations [shots, m], drawing from `generator` (a torch CPU generator) in the reference sampler's
    order: final spins (traced emitter), photon orders, then one multinomial per step and stream."""
    import torch
    U = np.asarray(U, dtype=np.complex128)
    m = U.shape[0]
    ops = np.asarray(ops, dtype=np.complex128)
    n, L, chi, _ = ops.shape
    if final is None:
        pf = torch.as_tensor(final_distribution(ops, s0)).clamp_min(0)
        fid = torch.multinomial(pf / pf.sum(), shots, replacement=True, generator=generator)
        finals = np.eye(chi)
    else:
        fid = torch.zeros(shots, dtype=torch.long)
        finals = np.asarray(final, dtype=np.complex128)[None]
    sigma = torch.argsort(torch.rand((shots, n), generator=generator), dim=1)
    rows = np.zeros((shots, n), dtype=np.int64)
    for k in range(1, n + 1):
        w = np.zeros((shots, m))
        for s in range(shots):
            T = sorted(sigma[s, :k].tolist())
            w[s] = candidate_weights(U, ops, modes, s0, finals[int(fid[s])], T, rows[s, :k - 1])
        wt = torch.as_tensor(w).clamp_min(0)
        wt = wt / wt.sum(dim=1, keepdim=True)
        rows[:, k - 1] = torch.multinomial(wt, 1, generator=generator).squeeze(1).numpy()
    occ = np.zeros((shots, m), dtype=np.int64)
    for j in range(n):
        np.add.at(occ, (np.arange(shots), rows[:, j]), 1)
    return occ


def matrix_weights(U, colmode, rows, s0, mats, f) -> np.ndarray:
    """w(rho) of one stream from given pure terms (emitter_reference.py:280-305, restated): colmode [k, L]
    input modes of the placed photons (sorted slots), rows the k - 1 chosen rows, s0 [R, chi],
    mats [R, k, L, chi, chi], f [R, chi].  Glynn sum over all delta in {+1} x {-1, +1}^(k-2) at once."""
    U = np.asarray(U, dtype=np.complex128)
    m = U.shape[0]
    colmode = np.asarray(colmode)
    k, L = colmode.shape
    kk = len(rows)
    if kk:
        grid = (np.array(list(itertools.product((1.0, -1.0), repeat=kk - 1))) if kk > 1
                else np.zeros((1, 0)))
        deltas = np.concatenate([np.ones((grid.shape[0], 1)), grid], axis=1)            # [D, kk]
        cs = np.einsum("di,ijl->djl", deltas, U[np.asarray(rows, dtype=np.int64)][:, colmode])
        sign = deltas.prod(axis=1)
        norm = 2.0 ** (-(kk - 1))
    else:
        cs, sign, norm = np.ones((1, k, L), dtype=np.complex128), np.ones(1), 1.0
    w = np.zeros(m)
    for e in range(np.asarray(s0).shape[0]):
        M = np.asarray(mats[e], dtype=np.complex128)
        G = np.einsum("djl,jlts->djts", cs, M)                                         # [D, k, chi, chi]
        D = G.shape[0]
        q = [None] * k
        u = np.broadcast_to(np.conj(np.asarray(f[e], dtype=np.complex128)), (D, M.shape[-1]))
        for c in range(k - 1, -1, -1):
            q[c] = u
            u = np.einsum("ds,dst->dt", u, G[:, c])
        v = np.broadcast_to(np.asarray(s0[e], dtype=np.complex128), (D, M.shape[-1]))
        t = np.zeros((k, L), dtype=np.complex128)
        for c in range(k):
            t[c] = np.einsum("d,dt,lts,ds->l", sign, q[c], M[c], v)
            v = np.einsum("dts,ds->dt", G[:, c], v)
        amp = (U[:, colmode] * (norm * t)[None]).sum(axis=(1, 2))
        w += np.abs(amp) ** 2
    return w
