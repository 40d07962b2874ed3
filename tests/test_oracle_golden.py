"""The CPU oracle against the golden vectors recorded from the reference implementation
(tests/golden/make_golden.py): Triton's Philox draws, cofactors of blocks with repeated rows (FP64 and
the reference's x87 long-double emulation), step amplitudes, and whole chains drawn by the reference."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O

PHILOX = np.load(os.path.join(GOLDEN, "philox.npz"))
STEPS = np.load(os.path.join(GOLDEN, "steps.npz"))
CHAINS = np.load(os.path.join(GOLDEN, "chains.npz"))


def test_philox_matches_triton_rand_bit_for_bit():
    for i, seed in enumerate(PHILOX["seeds"].tolist()):
        mine = np.array([O.triton_rand(seed, j) for j in range(PHILOX["rand_bits"].shape[1])], dtype=np.float32)
        assert np.array_equal(mine.view(np.uint32), PHILOX["rand_bits"][i])


def test_draw_uniforms_match_the_reference_draw_kernel():
    for i, seed in enumerate(PHILOX["seeds"].tolist()):
        u = O.uniforms([seed], PHILOX["uniforms"].shape[1])[:, 0]
        assert np.array_equal(u.view(np.uint64), PHILOX["uniforms"][i].view(np.uint64))


@pytest.mark.parametrize("i", range(len(STEPS["K1"])))
def test_cofactors_match_the_reference_sums(i):
    K1 = int(STEPS["K1"][i])
    K = K1 + 1
    B = STEPS["blocks"][i, :K1, :K]
    rows = STEPS["rows"][i, :K1]
    P, T = O.cofactors(B, rows)
    ref = STEPS["P_f64"][i, :K]
    scale = np.abs(ref).max()
    assert T == int(STEPS["addends"][i])
    assert np.abs(P - ref).max() <= 1e-13 * scale
    Pl, Tl = O.cofactors(B, rows, precision="ld")
    assert Tl == T
    assert np.abs(Pl - STEPS["P_ld"][i, :K]).max() <= 1e-14 * scale
    if K1 <= 9:
        R = O.ryser_cofactors(B)
        assert np.abs(P - R).max() <= 1e-12 * np.abs(R).max()


def test_step_weights_match_the_reference_step_amplitudes():
    U8 = STEPS["U8"]
    for rows, cols, amp in zip(STEPS["step_rows"], STEPS["step_cols"], STEPS["step_amps"]):
        rows = rows[rows >= 0]
        cols = cols[cols >= 0]
        _, w, _ = O.step(U8, rows, cols, 0.5)
        ref = np.abs(amp) ** 2
        assert np.abs(w - ref).max() <= 1e-13 * ref.max()


def test_addend_counts_follow_the_closed_form():
    assert O.addends([0, 1, 2, 3, 4]) == 16              # collision-free: 2^(K1 - 1)
    assert O.addends([2, 2, 2, 2]) == 5                  # one mode 4 times: prod(s + 1)
    assert O.addends([1, 1, 0]) == 3                     # (2 + 1) * (1 + 1) / 2
    assert O.addends([]) == 1


CHAIN_NAMES = sorted({k.split("__")[0] for k in CHAINS.files if k.endswith("__rows")})


@pytest.mark.parametrize("name", CHAIN_NAMES)
def test_oracle_chain_reproduces_the_reference_draws(name):
    """Same sigma, same per-step seeds -> the oracle picks exactly the rows the reference's sampler picked."""
    U = CHAINS[f"{name}__U"]
    in_modes = CHAINS[f"{name}__in_modes"].tolist()
    m, Bn, shots = CHAINS[f"{name}__meta"][:3].tolist()
    sig = CHAINS[f"{name}__sigma"]
    seeds = CHAINS[f"{name}__seeds"]
    S = Bn * shots
    A = U[:, :, in_modes]
    dp = np.repeat(np.arange(Bn), shots)
    out = O.chain(A, dp, sig, O.uniforms(seeds, S))
    assert np.array_equal(out["rows"], CHAINS[f"{name}__rows"])
    assert np.array_equal(O.occupations(out["rows"], m), CHAINS[f"{name}__occ"])
    assert out["gap"].min() > 1e-9                        # no draw near a CDF step: the comparison is meaningful


def test_long_double_chain_agrees_with_the_fp64_chain():
    U = O.haar_unitary(16, 7)
    A = U[:, :8]
    rng = np.random.default_rng(1)
    S = 6
    sig = np.argsort(rng.random((S, 8)), axis=1)
    u = rng.random((S, 8))
    a = O.chain(A, np.zeros(S, np.int64), sig, u, marg=True)
    b = O.chain(A, np.zeros(S, np.int64), sig, u, precision="ld", marg=True)
    assert np.array_equal(a["rows"], b["rows"])
    assert np.abs(a["marg"] - b["marg"]).max() <= 1e-12
    assert np.array_equal(a["addends"], b["addends"])


SLOS = np.load(os.path.join(GOLDEN, "slos.npz"))
SLOS_CASES = sorted({k.split("__")[0] for k in SLOS.files})


@pytest.mark.parametrize("name", SLOS_CASES)
def test_exact_distributions_match_the_reference_slos(name):
    """The oracle's exact output laws (Ryser enumeration; the lossy / x-model mixture) against the
    probabilities of the reference's SLOS kernel on the same circuits: every outcome within 1e-12, the
    same support.  These laws are the ones the histogram tests measure their TVD against."""
    m, seed, eta, x = SLOS[f"{name}__meta"].tolist()
    modes = SLOS[f"{name}__modes"].tolist()
    U = O.haar_unitary(int(m), int(seed))
    if eta < 0 and x < 0:
        dist = O.exact_distribution(U, modes)
    else:
        dist = O.imperfect_distribution(U, modes, 1.0 if eta < 0 else eta, 1.0 if x < 0 else x)
    ref = {tuple(int(v) for v in st): float(p) for st, p in zip(SLOS[f"{name}__states"], SLOS[f"{name}__probs"])}
    keys = set(ref) | {k for k, p in dist.items() if p > 1e-15}
    assert max(abs(dist.get(k, 0.0) - ref.get(k, 0.0)) for k in keys) <= 1e-12
    assert abs(sum(ref.values()) - 1.0) <= 1e-12
