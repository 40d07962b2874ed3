"""Adaptive sampling on the GPU (pe_fock_chain_adaptive through the C ABI): forced prefixes and avoided
modes against the reference's recorded draws (tests/golden/adaptive.npz), against the oracle's
restatement of the reference's early-abort chain on larger random cases, and the law of the survivors
against the exact output distribution.  Picks are bit-exact in the FP64 form; the mixed form returns the
FP64 form's picks (its guard band redoes ambiguous draws in FP64)."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from photonic_engines_b200.clifford import fock_sample
from photonic_engines_b200.clifford.kernels import chain_adaptive, pack_instances
from test_adaptive_cpu import CASES, case

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("name", CASES)
def test_fock_sample_reproduces_the_reference_adaptive_draws(name, precision):
    c = case(name)
    U = torch.as_tensor(c["U"], device=DEV)
    occ, ids = fock_sample(U if c["Bn"] > 1 else U[0], list(c["in_modes"]), c["shots"],
                           generator=torch.Generator().manual_seed(c["gseed"]), prefix=c["prefix_l"],
                           avoid=c["avoid_l"], keep_ids=True, max_streams=c["max_streams"], precision=precision)
    assert (occ.cpu().numpy() == c["occ"]).all()
    assert (ids.cpu().numpy() == c["ids"]).all()


def _random_case(seed, m, n, S, c0, n_avoid, Bn=1, max_streams=1 << 18):
    rng = np.random.default_rng(seed)
    U = np.stack([O.haar_unitary(m, seed * 10 + b) for b in range(Bn)])
    in_modes = list(range(n))
    dp = np.repeat(np.arange(Bn), S // Bn)
    sigma = np.stack([rng.permutation(n) for _ in range(S)])
    pre = rng.integers(0, m, size=(Bn, c0))
    pre_rows = pre[dp]
    seeds = rng.integers(0, 2 ** 31 - 1, size=(-(-S // max_streams), n))
    avoid = sorted(set(rng.choice(m, size=n_avoid, replace=False).tolist())) if n_avoid else None
    return U, in_modes, dp, sigma, pre_rows, seeds, np.arange(S) // max_streams, np.arange(S) % max_streams, avoid


@pytest.mark.parametrize(("m", "n", "S", "c0", "n_avoid", "mode", "precision", "max_streams"), [
    (16, 8, 300, 2, 3, "cta", "f64", 1 << 18),
    (16, 8, 300, 2, 3, "warp", "f64", 1 << 18),
    (16, 8, 300, 2, 3, "cta", "mixed", 1 << 18),
    (16, 8, 300, 2, 3, "warp", "mixed", 100),
    (24, 12, 120, 3, 4, "cta", "f64", 50),
    (24, 12, 120, 0, 4, "warp", "f64", 1 << 18),
    (20, 10, 200, 4, 0, "cta", "f64", 1 << 18),
    (30, 18, 40, 2, 5, "cta", "f64", 1 << 18),
    (30, 18, 40, 2, 5, "cta", "mixed", 1 << 18),
])
def test_adaptive_chains_match_the_oracle(m, n, S, c0, n_avoid, mode, precision, max_streams):
    U, in_modes, dp, sigma, pre_rows, seeds, seed_row, off0, avoid = _random_case(m * 7 + n, m, n, S, c0, n_avoid,
                                                                                  max_streams=max_streams)
    want_rows, want_alive = O.adaptive_chains(U[:, :, in_modes], dp, sigma, pre_rows, seeds, seed_row, off0, avoid)
    acol, inst_off, inst_m, inst_n = pack_instances(torch.as_tensor(U, device=DEV), in_modes)
    rows = torch.zeros(S, n, dtype=torch.int64, device=DEV)
    rows[:, :c0] = torch.as_tensor(pre_rows, device=DEV)
    mask = None
    if avoid:
        mask = torch.zeros(m, dtype=torch.uint8, device=DEV)
        mask[avoid] = 1
    rows, occ, alive = chain_adaptive(acol, inst_off, inst_m, inst_n, dp, sigma, rows, c0, avoid=mask, seeds=seeds,
                                      seed_row=seed_row, rng_off=off0, precision=precision, mode=mode)
    alive = alive.cpu().numpy()
    rows = rows.cpu().numpy()
    assert (alive == want_alive).all()
    assert (rows[alive] == want_rows[alive]).all()
    occ = occ.cpu().numpy()
    assert (occ[alive] == O.occupations(want_rows[alive], m)).all()
    assert (occ[~alive] == 0).all()


def test_a_split_adaptive_chain_matches_the_oracle():
    """Few long streams: the heavy steps spread over several CTAs per stream, one launch per step."""
    m, n, S, c0 = 40, 20, 6, 2
    U, in_modes, dp, sigma, pre_rows, seeds, seed_row, off0, avoid = _random_case(77, m, n, S, c0, 6)
    want_rows, want_alive = O.adaptive_chains(U[:, :, in_modes], dp, sigma, pre_rows, seeds, seed_row, off0, avoid)
    acol, inst_off, inst_m, inst_n = pack_instances(torch.as_tensor(U, device=DEV), in_modes)
    for split in [(12, 8), (14, 3)]:
        rows = torch.zeros(S, n, dtype=torch.int64, device=DEV)
        rows[:, :c0] = torch.as_tensor(pre_rows, device=DEV)
        mask = torch.zeros(m, dtype=torch.uint8, device=DEV)
        mask[avoid] = 1
        rows, occ, alive = chain_adaptive(acol, inst_off, inst_m, inst_n, dp, sigma, rows, c0, avoid=mask,
                                          seeds=seeds, seed_row=seed_row, rng_off=off0, split=split, mode="cta")
        alive = alive.cpu().numpy()
        assert (alive == want_alive).all(), split
        assert (rows.cpu().numpy()[alive] == want_rows[alive]).all(), split


def test_supplied_uniforms_with_a_prefix_match_the_oracle():
    m, n, S, c0 = 12, 7, 64, 3
    rng = np.random.default_rng(5)
    U = O.haar_unitary(m, 5)[None]
    sigma = np.stack([rng.permutation(n) for _ in range(S)])
    pre_rows = np.tile(np.array([4, 4, 9]), (S, 1))
    u = rng.random((S, n))
    want = np.zeros((S, n), dtype=np.int64)
    want[:, :c0] = pre_rows
    for s in range(S):
        for k in range(c0 + 1, n + 1):
            want[s, k - 1] = O.step(U[0][:, :n], want[s, :k - 1], sigma[s, :k], u[s, k - 1])[0]
    acol, inst_off, inst_m, inst_n = pack_instances(torch.as_tensor(U, device=DEV), list(range(n)))
    rows = torch.zeros(S, n, dtype=torch.int64, device=DEV)
    rows[:, :c0] = torch.as_tensor(pre_rows, device=DEV)
    rows, occ, alive = chain_adaptive(acol, inst_off, inst_m, inst_n, np.zeros(S), sigma, rows, c0, uniforms=u)
    assert bool(alive.all())
    assert (rows.cpu().numpy() == want).all()


def test_early_abort_keeps_the_conditional_law():
    """prefix=[3], avoid=[3]: every survivor has exactly one photon in mode 3, the survival fraction is
    P(N_3 = 1) / E[N_3], and the survivors follow the exact law conditioned on N_3 = 1 (the reference's
    tests/test_adaptive.py:315-327 claim, checked here against the exact output distribution)."""
    U = O.haar_unitary(5, 31)
    in_modes = [0, 1, 2]
    dist = O.exact_distribution(U, in_modes)
    P = sum(p for o, p in dist.items() if o[3] == 1)
    T = sum(p * o[3] for o, p in dist.items())
    shots = 40000
    kept = fock_sample(torch.as_tensor(U, device=DEV), in_modes, shots,
                       generator=torch.Generator(device=DEV).manual_seed(2), prefix=[3], avoid=[3]).cpu().numpy()
    assert kept.shape[1] == 5 and (kept.sum(1) == 3).all() and (kept[:, 3] == 1).all()
    ratio = P / T
    assert abs(kept.shape[0] / shots - ratio) < 4 * math.sqrt(ratio * (1 - ratio) / shots) + 1 / shots
    cond = {o: p / P for o, p in dist.items() if o[3] == 1}
    tvd, floor = O.tvd_and_floor(cond, kept)
    assert tvd < 2.5 * floor, (tvd, floor)


def test_a_forced_prefix_gives_the_conditional_law_at_acceptance():
    """prefix=[1, 3] without avoid, keeping draws with no further photon on modes 1 and 3: the exact law
    conditioned on (N_1, N_3) = (1, 1) (the reference's tests/test_adaptive.py:194-212)."""
    U = O.haar_unitary(5, 14)
    in_modes = [0, 1, 2, 4]
    dist = O.exact_distribution(U, in_modes)
    shots = 40000
    smp = fock_sample(torch.as_tensor(U, device=DEV), in_modes, shots,
                      generator=torch.Generator(device=DEV).manual_seed(4), prefix=[1, 3]).cpu().numpy()
    assert (smp.sum(1) == 4).all() and (smp[:, 1] >= 1).all() and (smp[:, 3] >= 1).all()
    keep = (smp[:, 1] == 1) & (smp[:, 3] == 1)
    P = sum(p for o, p in dist.items() if o[1] == 1 and o[3] == 1)
    T = sum(p * o[1] * o[3] for o, p in dist.items())
    ratio = P / T
    assert abs(keep.mean() - ratio) < 4 * math.sqrt(ratio * (1 - ratio) / shots) + 1 / shots
    cond = {o: p / P for o, p in dist.items() if o[1] == 1 and o[3] == 1}
    tvd, floor = O.tvd_and_floor(cond, smp[keep])
    assert tvd < 2.5 * floor, (tvd, floor)
