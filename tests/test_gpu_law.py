"""The sampled LAW at sizes where no exact distribution can be enumerated: closed-form first and second
moments of the output occupations, checked with Bonferroni-corrected z-scores through the public
`fock_sample`, in every precision form.

For n single photons in distinct input modes J of an m-mode interferometer U (indistinguishable, lossless):
    mu_a          = sum_{j in J} |U_aj|^2
    E[n_a n_b]    = mu_a mu_b + |M_ab|^2 - 2 W_ab   (a != b)
    E[n_a^2]      = 2 mu_a^2 - 2 W_aa + mu_a
with M_ab = sum_{j in J} U_aj conj(U_bj) and W_ab = sum_{j in J} |U_aj|^2 |U_bj|^2 (two-photon terms of
the permanent expansion).  The reference checks its large-n samplers the same way
(tests/clifford/check_large_n.py:100-140).  Distinguishable photons would give mu_a mu_b - W_ab instead;
the power checks below make sure the test tells the two laws apart."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from photonic_engines_b200.clifford import fock_sample

pytestmark = pytest.mark.gpu
DEV = "cuda"
ALPHA = 1e-3                    # family-wise false-alarm rate of one test


def _z_threshold(count: int) -> float:
    """Two-sided normal quantile at ALPHA / count (Bonferroni)."""
    p = ALPHA / count
    lo, hi = 0.0, 40.0
    for _ in range(200):                      # bisection on the normal tail: erfc(z / sqrt 2) = p
        mid = 0.5 * (lo + hi)
        if math.erfc(mid / math.sqrt(2.0)) > p:
            lo = mid
        else:
            hi = mid
    return hi


def _moments(U, J):
    A = U[:, J]
    P = np.abs(A) ** 2
    mu = P.sum(1)
    M = A @ A.conj().T
    W = P @ P.T
    second = mu[:, None] * mu[None, :] + np.abs(M) ** 2 - 2 * W
    second[np.diag_indices_from(second)] = 2 * mu ** 2 - 2 * np.diag(W) + mu
    classical = mu[:, None] * mu[None, :] - W
    classical[np.diag_indices_from(classical)] = mu ** 2 - np.diag(W) + mu
    return mu, second, classical


def _pair_z(occ, pairs, expect):
    x = occ[:, pairs[:, 0]] * occ[:, pairs[:, 1]]
    se = x.std(0, ddof=1) / math.sqrt(x.shape[0])
    return (x.mean(0) - expect[pairs[:, 0], pairs[:, 1]]) / np.maximum(se, 1e-300)


def _sample(U, n, shots, precision, seed):
    out = []
    g = torch.Generator(device=DEV).manual_seed(seed)
    Ut = torch.tensor(U, device=DEV)
    for c in range(0, shots, 4000):
        out.append(fock_sample(Ut, list(range(n)), min(4000, shots - c), generator=g, precision=precision).cpu())
    return torch.cat(out).numpy().astype(np.float64)


@pytest.mark.parametrize("precision", ["f64", "mixed", "compensated"])
def test_moments_at_n20_m400(precision):
    """The headline workload's shape: n = 20 photons in m = 400 modes, 24 000 samples.  First moments of
    all 400 modes and second moments of 200 pairs (100 off-diagonal pairs with the largest two-photon
    interference term |M_ab|^2 - W_ab and 100 diagonal ones), each within the Bonferroni threshold."""
    n, m, shots = 20, 400, 24000
    U = O.haar_unitary(m, 4242)
    mu, second, _ = _moments(U, list(range(n)))
    occ = _sample(U, n, shots, precision, 11)
    assert (occ.sum(1) == n).all()
    z1 = (occ.mean(0) - mu) / np.maximum(occ.std(0, ddof=1) / math.sqrt(shots), 1e-300)
    zt = _z_threshold(m + 200)
    assert np.abs(z1).max() < zt, (np.abs(z1).max(), zt)
    A = U[:, :n]
    D = np.abs(A @ A.conj().T) ** 2 - (np.abs(A) ** 2) @ (np.abs(A) ** 2).T
    iu = np.triu_indices(m, 1)
    top = np.argsort(-D[iu])[:100]
    pairs = np.concatenate([np.stack([iu[0][top], iu[1][top]], 1),
                            np.stack([np.argsort(-mu)[:100]] * 2, 1)])
    z2 = _pair_z(occ, pairs, second)
    assert np.abs(z2).max() < zt, (np.abs(z2).max(), zt)


@pytest.mark.parametrize("precision", ["f64", "compensated"])
def test_moments_tell_bosons_from_distinguishable_photons(precision):
    """Power of the moment test: n = 12 photons in m = 36 modes (strong two-photon interference), 40 000
    samples.  The bosonic second moments pass the Bonferroni threshold over all pairs; the distinguishable
    law's second moments are rejected by a wide margin on the same samples."""
    n, m, shots = 12, 36, 40000
    U = O.haar_unitary(m, 99)
    mu, second, classical = _moments(U, list(range(n)))
    occ = _sample(U, n, shots, precision, 5)
    iu = np.triu_indices(m)
    pairs = np.stack(iu, 1)
    zt = _z_threshold(len(pairs))
    zb = _pair_z(occ, pairs, second)
    zc = _pair_z(occ, pairs, classical)
    assert np.abs(zb).max() < zt, (np.abs(zb).max(), zt)
    assert np.abs(zc).max() > 2 * zt, (np.abs(zc).max(), zt)
    assert float(np.mean(zb ** 2)) < 1.5 and float(np.mean(zc ** 2)) > 10.0
