"""Column sets for a forced prefix (adaptive sampling: `fock_sample(prefix=...)`).

The chain is exact given the SET of input columns its first c steps use: rows_{<=c} | T ~ |per(A[rows, T])|^2
with T uniform among the c-subsets (photonic_engines/clifford/sampler.py:26-33).  Forcing the first c rows
onto `prefix` therefore draws T with weight |per(A[prefix, T])|^2, and the chain continues at step c + 1.

With the prefix's distinct modes b_1..b_L and multiplicities p = (p_1..p_L),
per(A[prefix, T]) = p! [x^p] prod_{j in T} (sum_l A[b_l, j] x_l), so T is drawn column by column without
enumerating the C(n, c) subsets (sampler.py:264-364, `prefix_columns` / `prefix_columns_many`).  Here the
recursion is written with D x D operators on the coefficient vectors (D = prod (p_l + 1), multi-indices
flattened row-major, degrees above p dropped):

    R_l          raises the degree of x_l by one (the coefficient at a moves to a + e_l)
    M_j          = sum_l A[b_l, j] R_l            multiplication by column j's linear form
    F_n          = e_0 e_0^H,  F_j = F_{j+1} + M_j F_{j+1} M_j^H
                                                  (sum over the subsets T' of columns j.. of c_T' c_T'^H)
    mass(v, F)   = sum_{a,b} v_a conj(v_b) F[p - a, p - b]
                                                  (= sum_T' |[x^p] v * c_T'|^2; p - a is the reversed flat index)

and column j joins the set with probability mass(M_j g, F_{j+1}) / (mass(M_j g, F_{j+1}) + mass(g, F_{j+1})),
g the polynomial of the columns taken so far — one float64 uniform per stream per column, drawn from the
caller's generator in the reference's order, so a seeded generator gives the reference's column sets.
"""
from __future__ import annotations

import itertools
import math

import torch


def _shape_of(prefix) -> tuple[list[int], list[int]]:
    """(modes, multiplicities) of a prefix, ordered by decreasing multiplicity then mode (the order in
    which circuits of one multiplicity shape line up, sampler.py:326)."""
    pre = [int(b) for b in prefix]
    cnt = sorted(((pre.count(b), b) for b in set(pre)), key=lambda x: (-x[0], x[1]))
    return [b for _, b in cnt], [c for c, _ in cnt]


def _raise_ops(p: list[int], device) -> torch.Tensor:
    """R [L, D, D] complex128: R[l] maps the coefficient at multi-index a to a + e_l (dropped past p_l)."""
    dims = [c + 1 for c in p]
    D = math.prod(dims)
    L = len(p)
    R = torch.zeros(L, D, D, dtype=torch.complex128)
    strides = [math.prod(dims[l + 1:]) for l in range(L)]
    for flat, a in enumerate(itertools.product(*[range(d) for d in dims])):
        for l in range(L):
            if a[l] < p[l]:
                R[l, flat + strides[l], flat] = 1.0
    return R.to(device)


def prefix_columns_many(A: torch.Tensor, prefixes, dp: torch.Tensor, generator=None) -> torch.Tensor:
    """bool [S, n]: stream s draws a column set of circuit dp[s] with weight |per(A[dp[s]][prefix, T])|^2.

    A [G, m, n] (the input columns of G circuits), prefixes: G lists of c output modes sharing one
    multiplicity shape (sampler.py:313-364).  Every column decision draws torch.rand(S, float64) from
    `generator` (on the generator's device) in column order.
    """
    A = A.to(torch.complex128)
    G, _, n = A.shape
    dev = A.device
    dp = torch.as_tensor(dp, dtype=torch.int64, device=dev)
    S = dp.shape[0]
    shapes = [_shape_of(pre) for pre in prefixes]
    p = shapes[0][1]
    if any(mult != p for _, mult in shapes):
        raise ValueError("prefix_columns_many: the prefixes must share one multiplicity shape")
    modes = torch.tensor([md for md, _ in shapes], dtype=torch.int64, device=dev)            # [G, L]
    B = torch.gather(A, 1, modes[:, :, None].expand(G, len(p), n))                         # [G, L, n]
    R = _raise_ops(p, dev)                                                                   # [L, D, D]
    D = R.shape[-1]
    M = torch.einsum("gln,lab->gnab", B, R)                                                  # [G, n, D, D]
    F = [None] * (n + 1)
    F[n] = torch.zeros(G, D, D, dtype=torch.complex128, device=dev)
    F[n][:, 0, 0] = 1.0
    for j in range(n - 1, -1, -1):
        Mj = M[:, j]
        F[j] = F[j + 1] + Mj @ F[j + 1] @ Mj.conj().transpose(-1, -2)
    gdev = generator.device if generator is not None else dev
    g = torch.zeros(S, D, dtype=torch.complex128, device=dev)
    g[:, 0] = 1.0
    chosen = torch.zeros(S, n, dtype=torch.bool, device=dev)

    def mass(v, Fr):                                         # [S]: v^T Fr conj(v), Fr [S, D, D]
        return torch.einsum("sa,sab,sb->s", v, Fr, v.conj()).real.clamp_min(0.0)

    for j in range(n):
        Fr = F[j + 1].flip(-1).flip(-2)[dp]                  # F[p - a, p - b]: the flat index reversed
        g_in = torch.einsum("sab,sb->sa", M[dp, j], g)
        w_in, w_out = mass(g_in, Fr), mass(g, Fr)
        r = torch.rand(S, generator=generator, device=gdev, dtype=torch.float64).to(dev)
        take = r * (w_in + w_out) < w_in
        chosen[:, j] = take
        g = torch.where(take[:, None], g_in, g)
    return chosen


def prefix_columns(A: torch.Tensor, prefix, shots: int, generator=None) -> torch.Tensor:
    """bool [shots, n]: `shots` column sets of ONE circuit A [m, n] drawn with weight |per(A[prefix, T])|^2
    (sampler.py:264-310)."""
    return prefix_columns_many(A[None], [list(prefix)], torch.zeros(shots, dtype=torch.int64, device=A.device),
                               generator)


def prefix_subset_weights(A: torch.Tensor, prefix) -> tuple[torch.Tensor, torch.Tensor]:
    """The enumerated posterior of the column set (sampler.py:240-261): (subsets [C(n, c), c] int64,
    weights [G, C(n, c)] = |per(A[g][prefix, T])|^2).  A [G, m, n]; C(n, c) permanents, small cases only."""
    A = A.to(torch.complex128)
    n, c = A.shape[2], len(prefix)
    subs = torch.tensor(list(itertools.combinations(range(n), c)), dtype=torch.int64).reshape(-1, c)
    rows = torch.as_tensor(list(prefix), dtype=torch.int64, device=A.device)
    blocks = A[:, rows][:, :, subs.to(A.device)].permute(0, 2, 1, 3)                        # [G, C, c, c]
    per = _ryser(blocks)
    return subs, per.real ** 2 + per.imag ** 2


def _ryser(M: torch.Tensor) -> torch.Tensor:
    """Permanents of the trailing [c, c] blocks by Ryser's formula (c = 0 gives 1)."""
    c = M.shape[-1]
    if c == 0:
        return torch.ones(M.shape[:-2], dtype=M.dtype, device=M.device)
    tot = torch.zeros(M.shape[:-2], dtype=M.dtype, device=M.device)
    for mask in range(1, 1 << c):
        cols = [j for j in range(c) if mask >> j & 1]
        tot = tot + (-1.0) ** (c - len(cols)) * M[..., cols].sum(-1).prod(-1)
    return tot


def prefix_order(A: torch.Tensor, dp: torch.Tensor, n: int, prefix: torch.Tensor, generator=None) -> torch.Tensor:
    """The column order sigma [S, n] of a pass with a forced prefix (sampler.py:367-388): a uniform key per
    (stream, column), the key of the drawn prefix columns set to -1 so they sort first, circuits grouped
    by the multiplicity shape of their prefix (one batched draw per shape, in order of first circuit).
    A [G, m, n] input columns, dp [S], prefix [c] shared or [G, c] per circuit.  The key and the sort live
    on the generator's device (the reference's device when the generator is on U's device)."""
    dev = A.device
    gdev = generator.device if generator is not None else dev
    S = dp.shape[0]
    key = torch.rand(S, n, generator=generator, device=gdev)
    dp_g = dp.to(gdev)
    pre_of = (lambda g: prefix[g].tolist()) if prefix.dim() == 2 else (lambda g: prefix.tolist())
    groups: dict = {}
    for g in torch.unique(dp).tolist():
        pre = pre_of(g)
        shape = tuple(sorted((pre.count(b) for b in set(pre)), reverse=True))
        groups.setdefault(shape, []).append(g)
    for gs in groups.values():
        gs_t = torch.tensor(gs, dtype=torch.int64, device=gdev)
        ids = torch.nonzero(torch.isin(dp_g, gs_t))[:, 0]
        local = torch.searchsorted(gs_t, dp_g[ids])
        chosen = prefix_columns_many(A[gs_t.to(dev)], [pre_of(g) for g in gs], local.to(dev), generator).to(gdev)
        key[ids] = torch.where(chosen, torch.full_like(key[ids], -1.0), key[ids])
    return torch.argsort(key, dim=1).contiguous()
