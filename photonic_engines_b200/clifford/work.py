"""Algorithmic work of sampled chains, from their rows (the closed form of the collapsed sum).

At step k of a stream the collapsed Glynn sum over the k - 1 chosen rows has
    N_k = prod_groups (mult + 1), halved when some multiplicity is odd
terms (the reference's addend count, photonic_engines/clifford/variants.py:197-215 and
cofactors_triton.py:413-447), each a column-term update of k columns.  Per sample:
    W     = sum_k N_k k                       column-term updates
    FLOPs = 22 W + sum_k (8 m k + 2 m)        (column update 4, complex product 6, all-but-one
                                               accumulation 12 per column-term; marginal, |.|^2, scan)
    bytes = sum_k (16 m k + 16 k^2)           (gathered columns for the marginal + the cofactor block)
"""
from __future__ import annotations

import numpy as np


def chain_work(rows, m: int, nk=None) -> dict:
    """rows [S, n] ordered output modes (entries past nk[s] ignored) -> totals over the S chains:
    addends, column_terms W, flops, bytes, and per-step addends [n]."""
    rows = np.asarray(rows, dtype=np.int64)
    S, n = rows.shape
    nk = np.full(S, n) if nk is None else np.asarray(nk).reshape(-1)
    addends = 0
    W = 0
    flops = 0.0
    nbytes = 0.0
    per_step = np.zeros(n, dtype=np.float64)
    for k in range(1, n + 1):
        live = nk >= k
        cnt = int(live.sum())
        if cnt == 0:
            continue
        K1 = k - 1
        if K1 == 0:
            N = np.ones(cnt, dtype=np.int64)
        else:
            rs = np.sort(rows[live, :K1], axis=1)
            newgrp = np.ones_like(rs, dtype=bool)
            newgrp[:, 1:] = rs[:, 1:] != rs[:, :-1]
            gid = np.cumsum(newgrp, axis=1) - 1
            mult = np.zeros_like(rs)
            np.add.at(mult, (np.arange(cnt)[:, None], gid), 1)
            active = mult > 0
            has_odd = ((mult % 2 == 1) & active).any(axis=1)
            N = np.where(active, mult + 1, 1).prod(axis=1) // np.where(has_odd, 2, 1)
        addends += int(N.sum())
        W += int(N.sum()) * k
        per_step[k - 1] = float(N.sum())
        flops += 22.0 * float(N.sum()) * k + cnt * (8.0 * m * k + 2.0 * m)
        nbytes += cnt * (16.0 * m * k + 16.0 * k * k)
    return {"addends": addends, "column_terms": W, "flops": flops, "bytes": nbytes, "per_step": per_step}
