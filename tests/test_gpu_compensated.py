"""The compensated mixed form (precision="compensated"): FP32 Gray blocks in double-float arithmetic, held to
the 1e-6 marginal bound against the long-double oracle, and its picks equal to the FP64 form's.

Tolerances: cofactors and marginals within COMP_TOL = 1e-6 relative (normwise, per chain and step) of the
long-double oracle — the bound the compensated form is built for; its measured error is about 1e-10 on
distinct rows, and the tests also hold it to COMP_TIGHT = 1e-8 there (1e-7 on heavily repeated rows, where
the collapsed sum's binomial weights cancel strongly and the double-float pair's ~2^-44 per term shows) so
that a lost compensation (which lands at 1e-5) cannot hide under the bound.  Picks: identical to the FP64
form's wherever the oracle's draw lies farther than 1e-11 of the total weight from every CDF step."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from photonic_engines_b200.clifford import fock_sample, laplace_cofactors_rows, sample_chains

pytestmark = pytest.mark.gpu
DEV = "cuda"
COMP_TOL = 1e-6
COMP_TIGHT = 1e-8
COMP_TIGHT_COLLISIONS = 1e-7


def _rel(a, b):
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / scale) if scale > 0 else float(np.abs(a).max())


def _random_chains(n, m, S, seed):
    U = O.haar_unitary(m, seed)
    rng = np.random.default_rng(seed)
    sig = np.argsort(rng.random((S, n)), axis=1)
    u = rng.random((S, n))
    return U, sig, u


@pytest.mark.parametrize("K1,collide", [(3, False), (7, True), (11, False), (15, True), (19, False), (23, True)])
def test_compensated_cofactors_match_long_double(K1, collide):
    """Random complex blocks, distinct rows or repeated ones (the collapsed 2020 sum), against the
    long-double oracle."""
    rng = np.random.default_rng(300 + K1)
    K, S, m = K1 + 1, 3, 3 * (K1 + 1)
    A = (rng.normal(size=(S, m, K)) + 1j * rng.normal(size=(S, m, K))) / np.sqrt(2 * m)
    rows = rng.integers(0, max(2, K1 // 3), size=(S, K1)) if collide else np.stack(
        [rng.choice(m, K1, replace=False) for _ in range(S)])
    P = laplace_cofactors_rows(torch.tensor(A, device=DEV), torch.tensor(rows, device=DEV),
                               precision="compensated").cpu().numpy()
    for s in range(S):
        ref, _ = O.cofactors(A[s][rows[s]], rows[s], precision="ld")
        err = _rel(P[s], ref)
        assert err <= (COMP_TIGHT_COLLISIONS if collide else COMP_TIGHT), (s, err)


@pytest.mark.parametrize("tpl", [0, 2])
def test_compensated_chains_meet_the_bound_at_n20_m400(tpl):
    """The headline workload's shape (n = 20, m = 400): 12 chains with supplied uniforms against the
    long-double oracle — every marginal of every step within 1e-6 (COMP_TOL), picks equal to the FP64
    form's and the oracle's."""
    n, m, S = 20, 400, 12
    U, sig, u = _random_chains(n, m, S, 2020)
    ref = O.chain(U[:, :n], np.zeros(S, np.int64), sig, u, precision="ld", marg=True, threads=S)
    Ut = torch.tensor(U, device=DEV)
    cmp_ = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, precision="compensated", tpl=tpl)
    f64 = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True)
    far = (ref["gap"] > 1e-11).all(axis=1)
    assert far.sum() >= S - 1
    rows = cmp_["rows"].cpu().numpy()
    assert np.array_equal(rows, f64["rows"].cpu().numpy())
    assert np.array_equal(rows[far], ref["rows"][far])
    mc = cmp_["marg"].cpu().numpy()
    worst = 0.0
    for s in np.nonzero(far)[0]:
        for k in range(n):
            worst = max(worst, _rel(mc[s, k], ref["marg"][s, k]))
    assert worst <= COMP_TIGHT, worst
    assert worst <= COMP_TOL


def test_compensated_error_by_step_up_to_28_photons():
    """n = 28, m = 784 (the deep-permanent configuration's shape), 3 chains: the compensated marginals
    against the FP64 form's at every step (FP64 is within 1e-10 of long double there), bounded by 1e-6
    at every k — the per-k error of the FP32 blocks stays flat instead of growing ~1.2x per column."""
    n, m, S = 28, 784, 3
    U, sig, u = _random_chains(n, m, S, 2828)
    Ut = torch.tensor(U, device=DEV)
    cmp_ = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, precision="compensated", split=None)
    f64 = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, split=None)
    assert torch.equal(cmp_["rows"], f64["rows"])
    mc, m64 = cmp_["marg"].cpu().numpy(), f64["marg"].cpu().numpy()
    per_k = [max(_rel(mc[s, k], m64[s, k]) for s in range(S)) for k in range(n)]
    assert max(per_k) <= COMP_TIGHT, per_k


@pytest.mark.parametrize("k_split,nch", [(9, 8), (14, 64)])
def test_compensated_split_steps_match_single_cta_chains(k_split, nch):
    n, m, S = 18, 60, 4
    U, sig, u = _random_chains(n, m, S, 181)
    Ut = torch.tensor(U, device=DEV)
    a = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, precision="compensated", split=False)
    b = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, precision="compensated",
                      split=(k_split, nch))
    assert torch.equal(a["rows"], b["rows"])
    ma, mb = a["marg"].cpu().numpy(), b["marg"].cpu().numpy()
    for s in range(S):
        for k in range(n):
            assert _rel(mb[s, k], ma[s, k]) <= COMP_TIGHT


def test_compensated_fock_sample_gives_the_fp64_samples():
    """Through the public entry point, lossless and lossy: the same generator gives the FP64 form's samples."""
    U = torch.tensor(O.haar_unitary(60, 12), device=DEV)
    for kw in ({}, {"loss": 0.7}, {"indist": 0.9}):
        a = fock_sample(U, list(range(12)), 300, generator=torch.Generator().manual_seed(8), **kw)
        b = fock_sample(U, list(range(12)), 300, generator=torch.Generator().manual_seed(8), precision="compensated",
                        **kw)
        assert torch.equal(a, b), kw
