"""Adaptive sampling (`fock_sample(prefix=, avoid=)`) on the host: the oracle's restatement of the reference's
forced-prefix / early-abort chain, the column-set draw of a forced prefix, and the argument checks.

Pinned on the reference's own outputs (tests/golden/adaptive.npz, made by make_golden.py): `_sample_streams`
rows and survivors and `fock_sample(..., keep_ids=True)` occupations (photonic_engines/clifford/sampler.py:
57-182, 367-460).  The column-set law follows the reference's tests/test_adaptive.py:230-260, 492-510."""
import math
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import oracle as O
from photonic_engines_b200.clifford import fock_sample, prefix_columns, prefix_columns_many, prefix_subset_weights
from photonic_engines_b200.clifford.prefix import prefix_order

ADAPT = np.load(os.path.join(GOLDEN, "adaptive.npz"))
CASES = sorted({k.split("__")[0] for k in ADAPT.files if k.endswith("__occ")})


def case(name):
    z = {k.split("__")[1]: ADAPT[k] for k in ADAPT.files if k.startswith(name + "__")}
    m, Bn, shots, gseed, useed, max_streams = (int(x) for x in z["meta"])
    S = Bn * shots
    dp = np.repeat(np.arange(Bn), shots)
    pre = z["prefix"]
    c0 = pre.shape[-1] if pre.size else 0
    pre_rows = np.zeros((S, 0), dtype=np.int64) if c0 == 0 else (pre[dp] if pre.ndim == 2 else np.tile(pre, (S, 1)))
    return dict(z, m=m, Bn=Bn, shots=shots, gseed=gseed, S=S, dp=dp, c0=c0, pre_rows=pre_rows,
                max_streams=max_streams, seed_row=np.arange(S) // max_streams, off0=np.arange(S) % max_streams,
                avoid_l=[int(r) for r in z["avoid"]] or None, prefix_l=pre.tolist() if c0 else None)


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_the_reference_adaptive_chains(name):
    c = case(name)
    rows, alive = O.adaptive_chains(c["U"][:, :, c["in_modes"]], c["dp"], c["sigma"], c["pre_rows"], c["seeds"],
                                    c["seed_row"], c["off0"], c["avoid_l"])
    assert (alive == c["alive"]).all()
    assert (rows[alive] == c["rows"][alive]).all()
    assert (O.occupations(rows[alive], c["m"]) == c["occ"]).all()
    assert (np.nonzero(alive)[0] == c["ids"]).all()


@pytest.mark.parametrize("name", [n for n in CASES if case(n)["c0"] > 0])
def test_prefix_order_reproduces_the_reference_column_orders(name):
    c = case(name)
    U = torch.as_tensor(c["U"])
    A = U[:, :, list(c["in_modes"])]
    gen = torch.Generator().manual_seed(c["gseed"])
    pre = torch.as_tensor(c["prefix"])
    n = len(c["in_modes"])
    sig = []
    for s0 in range(0, c["S"], c["max_streams"]):
        dpc = torch.as_tensor(c["dp"][s0:s0 + c["max_streams"]])
        sig.append(prefix_order(A, dpc, n, pre, gen))
        torch.randint(0, 2 ** 31 - 1, (n,), generator=gen)                 # the chunk's step seeds
    assert (torch.cat(sig).numpy() == c["sigma"]).all()


def _tvd_vs_enumerated(chosen, sub, w):
    ref = w / w.sum()
    index = {tuple(t): i for i, t in enumerate(sub.tolist())}
    emp = torch.zeros_like(ref)
    rows, cnt = torch.unique(chosen, dim=0, return_counts=True)
    for r, k in zip(rows, cnt.tolist(), strict=True):
        emp[index[tuple(torch.nonzero(r)[:, 0].tolist())]] = k / chosen.shape[0]
    floor = 0.5 * math.sqrt(2 / math.pi) * float((ref * (1 - ref) / chosen.shape[0]).sqrt().sum())
    return 0.5 * float((emp - ref).abs().sum()), floor


@pytest.mark.parametrize("prefix", [[5], [5, 5], [5, 2], [2, 5, 5, 11], [11, 11, 11, 2, 2]])
def test_prefix_columns_draw_the_enumerated_posterior(prefix):
    A = torch.as_tensor(O.haar_unitary(12, 3))[:, [0, 1, 3, 4, 6, 8, 9]]
    sub, w = prefix_subset_weights(A[None], prefix)
    chosen = prefix_columns(A, prefix, 30000, torch.Generator().manual_seed(1))
    assert chosen.sum(1).tolist() == [len(prefix)] * 30000
    tvd, floor = _tvd_vs_enumerated(chosen, sub, w[0])
    assert tvd < 2.5 * floor, (tvd, floor)


def test_batched_prefix_columns_draw_each_circuits_posterior():
    A = torch.stack([torch.as_tensor(O.haar_unitary(12, 40 + g))[:, [0, 1, 3, 4, 6, 8, 9]] for g in range(3)])
    prefixes = [[5, 5, 2], [11, 3, 11], [0, 7, 7]]
    per = 10000
    dp = torch.arange(3).repeat(per)
    chosen = prefix_columns_many(A, prefixes, dp, torch.Generator().manual_seed(3))
    for g in range(3):
        sub, w = prefix_subset_weights(A[g:g + 1], prefixes[g])
        tvd, floor = _tvd_vs_enumerated(chosen[dp == g], sub, w[0])
        assert tvd < 2.5 * floor, (g, tvd, floor)


def test_prefix_weights_sum_to_the_chance_of_the_prefix():
    """sum_T |per(A[prefix, T])|^2 / (c! C(n, c)) = P(first c photons of the chain read `prefix`, in order),
    checked against the exact output distribution: the chance that c photons drawn without replacement
    from an outcome land on the prefix modes in that order."""
    U = O.haar_unitary(5, 9)
    in_modes = [0, 1, 2]
    dist = O.exact_distribution(U, in_modes)
    A = torch.as_tensor(U[:, in_modes])
    for prefix in ([3], [3, 3], [1, 4]):
        _, w = prefix_subset_weights(A[None], prefix)
        c, n = len(prefix), len(in_modes)
        got = float(w.sum()) / (math.factorial(c) * math.comb(n, c))
        want = 0.0
        for occ, p in dist.items():
            left, q = list(occ), 1.0
            for j, b in enumerate(prefix):
                q *= left[b] / (n - j)
                left[b] -= 1
            want += p * q
        assert got == pytest.approx(want, rel=1e-10, abs=1e-14)


def test_prefix_columns_are_polynomial_in_the_prefix_length():
    """13 forced photons on 38 columns: C(38, 13) = 5e9 subsets, never enumerated."""
    A = torch.as_tensor(O.haar_unitary(76, 5))[:, :38]
    chosen = prefix_columns(A, [75] * 7 + [74] * 6, 4, torch.Generator().manual_seed(0))
    assert chosen.sum(1).tolist() == [13] * 4


def test_prefixes_of_different_shapes_are_refused_in_one_batch():
    A = torch.as_tensor(O.haar_unitary(6, 2))[:, :4]
    with pytest.raises(ValueError, match="multiplicity shape"):
        prefix_columns_many(torch.stack([A, A]), [[1, 1], [1, 2]], torch.tensor([0, 1]))


U6 = torch.as_tensor(O.haar_unitary(6, 13))


@pytest.mark.parametrize(("kw", "exc"), [({"prefix": [1], "loss": 0.5}, NotImplementedError),
                                         ({"avoid": [2], "indist": 0.9}, NotImplementedError),
                                         ({"prefix": [1], "backend": "exq"}, NotImplementedError),
                                         ({"prefix": [1, 2, 3, 4]}, ValueError),
                                         ({"prefix": [6]}, ValueError),
                                         ({"prefix": [-1]}, ValueError),
                                         ({"prefix": [[1], [2]]}, ValueError),
                                         ({"avoid": [7]}, ValueError)])
def test_bad_prefix_and_avoid_arguments_are_refused(kw, exc):
    with pytest.raises(exc):
        fock_sample(U6, [0, 1, 2], 4, generator=torch.Generator().manual_seed(0), **kw)
