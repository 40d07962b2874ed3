"""Chains of 33 to 64 photons on the GPU (the wide tiers: 40, 48, 56 and 64 columns, FP64, two-thread
lanes at 40 and four-thread lanes at 40 and beyond, 64-wide shared-memory tables), through the C ABI.

The oracle finishes such chains in seconds only when few distinct rows are chosen (the term count is the
product of multiplicity + 1 over the distinct rows), so the chains run in few modes: picks bit-exact with
the oracle's, marginals step by step against the long-double oracle.  A step with 34 distinct rows (2^33 terms, the planner's
second group per lane) is checked against a closed form: a bidiagonal block B[i][i] = a_i,
B[i][i + 1] = b_i has cofactors P_c = prod_{i < c} a_i prod_{i >= c} b_i, so its marginal and pick are
known exactly."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from photonic_engines_b200 import _native as N
from photonic_engines_b200.clifford import fock_sample, laplace_cofactors_rows, sample_chains
from photonic_engines_b200.clifford.kernels import chain_adaptive, pack_instances
from test_gpu_parity import _random_chains, _rel

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.mark.parametrize(("n", "m", "split", "tpl"), [(36, 8, False, 0), (38, 8, None, 4), (44, 7, False, 0),
                                                      (48, 6, None, 0), (64, 5, False, 0)])
def test_wide_chains_match_the_oracle(n, m, split, tpl):
    """Every step of the GPU's chains against the long-double oracle's step on the same history: the
    marginal within 50x the FP64 oracle's own distance from long double at that step (high multiplicities
    cancel: at k = 64 in 5 modes FP64 keeps ~3 digits), the pick equal wherever the draw is farther than
    twice that from every CDF step; and the chains bit-exact with the FP64 oracle's when no draw is close."""
    S = 4
    U, sig, u = _random_chains(n, m, S, 900 + n)
    in_modes = [i % m for i in range(n)]                      # n photons in m < n input modes
    A = U[:, in_modes]
    out = sample_chains(torch.tensor(U, device=DEV), in_modes, sig, uniforms=u, want_marg=True, split=split, tpl=tpl)
    rows, mg = out["rows"].cpu().numpy(), out["marg"].cpu().numpy()
    exact = 0
    for s in range(S):
        clear = True
        for k in range(1, n + 1):
            pick, w, gap = O.step(A, rows[s, :k - 1], sig[s, :k], u[s, k - 1], precision="ld")
            _, w64, _ = O.step(A, rows[s, :k - 1], sig[s, :k], u[s, k - 1], precision="f64")
            want = w / w.sum()
            tol = max(1e-10, 50 * _rel(w64 / w64.sum(), want))
            assert _rel(mg[s, k - 1], want) <= tol, (s, k)
            if gap > 2 * tol:
                assert rows[s, k - 1] == pick, (s, k)
            else:
                clear = False
        if clear:                                   # no draw near a CDF step: the FP64 oracle's chain
            ref = O.chain(A, np.zeros(1, np.int64), sig[s:s + 1], u[s:s + 1])
            assert np.array_equal(rows[s], ref["rows"][0])
            exact += 1
    assert exact >= S - 1


@pytest.mark.parametrize("K1", [35, 47, 63])
def test_wide_cofactor_steps_match_the_oracle(K1):
    """Repeated-row blocks of 36 to 64 columns over six distinct rows, against the long-double oracle,
    within 1e-9 or 100x the FP64 oracle's own distance from it (multiplicities near 10 cancel digits,
    and two FP64 summation orders land up to ~100x apart on one block)."""
    rng = np.random.default_rng(K1)
    K, S, m = K1 + 1, 3, 6
    A = rng.normal(size=(S, m, K)) + 1j * rng.normal(size=(S, m, K))
    rows = rng.integers(0, m, size=(S, K1))
    P = laplace_cofactors_rows(torch.tensor(A, device=DEV), torch.tensor(rows, device=DEV)).cpu().numpy()
    for s in range(S):
        ref, _ = O.cofactors(A[s][rows[s]], rows[s], precision="ld")
        r64, _ = O.cofactors(A[s][rows[s]], rows[s], precision="f64")
        assert _rel(P[s], ref) <= max(1e-9, 100 * _rel(r64, ref)), s


def test_a_step_with_34_distinct_rows_has_the_bidiagonal_marginal():
    """35 photons, 34 forced distinct rows 0..33 whose block is bidiagonal, the 35th step drawn by the
    GPU (2^33 terms: 33 active row groups, the last one halved; heavy steps split over the GPU): every
    pick equals the pick of the exact marginal."""
    n, c0 = 35, 34
    m = 48
    rng = np.random.default_rng(7)
    a = rng.uniform(0.5, 1.5, size=c0) * np.exp(1j * rng.uniform(0, 2 * np.pi, size=c0))
    b = rng.uniform(0.5, 1.5, size=c0) * np.exp(1j * rng.uniform(0, 2 * np.pi, size=c0))
    A = np.zeros((m, n), dtype=np.complex128)
    for i in range(c0):
        A[i, i], A[i, i + 1] = a[i], b[i]
    A[c0:] = (rng.normal(size=(m - c0, n)) + 1j * rng.normal(size=(m - c0, n))) / np.sqrt(n)
    P = np.array([np.prod(a[:c]) * np.prod(b[c:]) for c in range(n)])
    w = np.abs(A @ P) ** 2
    cw = np.cumsum(w)
    us = np.array([0.05, 0.45, 0.93])
    S = len(us)
    want = np.minimum((cw[None, :] < (us * cw[-1])[:, None]).sum(1), m - 1)
    gap = np.min(np.abs(cw[None, :] - (us * cw[-1])[:, None]), axis=1) / cw[-1]
    assert (gap > 1e-6).all()
    Uf = np.zeros((1, m, m), dtype=np.complex128)
    Uf[0, :, :n] = A
    acol, inst_off, inst_m, inst_n = pack_instances(torch.tensor(Uf, device=DEV), list(range(n)))
    cols = np.tile(np.arange(n), (S, 1))
    rows = torch.zeros(S, n, dtype=torch.int64, device=DEV)
    rows[:, :c0] = torch.arange(c0, device=DEV)
    u = np.zeros((S, n))
    u[:, c0] = us
    rows, occ, alive = chain_adaptive(acol, inst_off, inst_m, inst_n, np.zeros(S), cols, rows, c0, uniforms=u,
                                      split=(c0 + 1, 64))
    assert bool(alive.all())
    assert (rows.cpu().numpy()[:, c0] == want).all(), (rows.cpu().numpy()[:, c0], want)


def test_fock_sample_runs_40_photons_and_refuses_the_mixed_form():
    m, n = 10, 40
    U = torch.tensor(O.haar_unitary(m, 3), device=DEV)
    occ = fock_sample(U, [i % m for i in range(n)], 3, generator=torch.Generator(device=DEV).manual_seed(1))
    assert occ.shape == (3, m) and (occ.sum(1) == n).all()
    with pytest.raises(ValueError, match="mixed"):
        fock_sample(U, [i % m for i in range(n)], 3, precision="mixed")
    L = N.load()
    assert L.pe_split_slots(N.PRECISIONS["mixed"], 40, 0, 0) == N.PE_ERR_SIZE
    assert L.pe_split_slots(N.PRECISIONS["f64"], 40, 0, 0) > 0
