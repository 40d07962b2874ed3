"""Parity at the shapes of the benchmark configurations (the shapes the reference's own GPU checks use for
the same purpose, tests/clifford/check_cuda.py:38-50): the CUDA chains against the long-double oracle with
supplied uniforms, and the forms against each other through the public fock_sample.

  c3 shape  m = 900, chains of up to 30 of the 30 input columns (the lossy configuration's survivors)
  c4 shape  n = 28, m = 784, x-model indist 0.95 through fock_sample
  c5 shape  a sample of the 256 small circuits (m in {16, 24, 32, 48, 64}, n <= 12)

Tolerances as tests/test_gpu_parity.py: FP64 picks bit-exact where the oracle's draw lies farther than
1e-11 of the total weight from every CDF step, marginals within f64_tol(k); both FP32 forms' picks equal
to the FP64 form's; compensated marginals within 1e-8 (the 1e-6 bound with margin), plain mixed within
its envelope."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from photonic_engines_b200.clifford import fock_sample, sample_chains

pytestmark = pytest.mark.gpu
DEV = "cuda"


def f64_tol(k: int) -> float:
    return 1e-10 * max(1.0, 1.8 ** (k - 24))


def mixed_tol(k: int) -> float:
    return 2e-7 * 1.35 ** k


def _rel(a, b):
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / scale) if scale > 0 else float(np.abs(a).max())


@pytest.mark.parametrize("k", [24, 26])
def test_c3_shape_chains_match_the_long_double_oracle(k):
    """m = 900, 3 chains of k photons on k of the 30 input columns (as a lossy pass runs them)."""
    m, n_in, S = 900, 30, 3
    U = O.haar_unitary(m, 3001)
    rng = np.random.default_rng(900 + k)
    cols = np.sort(rng.choice(n_in, k, replace=False))
    sig = np.stack([cols[rng.permutation(k)] for _ in range(S)])          # column order per chain
    u = rng.random((S, k))
    ref = O.chain(U[:, :n_in], np.zeros(S, np.int64), sig, u, precision="ld", marg=True, threads=S)
    Ut = torch.tensor(U, device=DEV)
    out = {p: sample_chains(Ut, list(range(n_in)), sig, uniforms=u, want_marg=True, precision=p, split=None)
           for p in ("f64", "mixed", "compensated")}
    far = (ref["gap"] > 1e-11).all(axis=1)
    assert far.sum() >= 2
    rows64 = out["f64"]["rows"].cpu().numpy()
    assert np.array_equal(rows64[far], ref["rows"][far])
    for p in ("mixed", "compensated"):
        assert np.array_equal(out[p]["rows"].cpu().numpy(), rows64), p
    marg = {p: out[p]["marg"].cpu().numpy() for p in out}
    for s in np.nonzero(far)[0]:
        for j in range(k):
            assert _rel(marg["f64"][s, j], ref["marg"][s, j]) <= f64_tol(j + 1), (s, j)
            assert _rel(marg["compensated"][s, j], ref["marg"][s, j]) <= 1e-8, (s, j)
            assert _rel(marg["mixed"][s, j], ref["marg"][s, j]) <= mixed_tol(j + 1), (s, j)


def test_c3_shape_guard_band_keeps_fp64_picks_at_32_columns():
    """m = 900, 8 chains of 32 photons (the widest mixed tier, where the mixed form's CDF deviation is largest):
    the plain mixed form's picks equal the FP64 form's at every step (guard band per step)."""
    m, n, S = 900, 32, 8
    U = torch.tensor(O.haar_unitary(m, 3201), device=DEV)
    rng = np.random.default_rng(32)
    sig = np.argsort(rng.random((S, n)), axis=1)
    u = rng.random((S, n))
    a = sample_chains(U, list(range(n)), sig, uniforms=u, split=None)
    b = sample_chains(U, list(range(n)), sig, uniforms=u, split=None, precision="mixed")
    assert torch.equal(a["rows"], b["rows"])


def test_c4_shape_forms_give_the_same_samples_through_fock_sample():
    """n = 28, m = 784, x-model indist 0.95, 24 shots from one seeded generator: the FP64, mixed and
    compensated forms return the same occupations (host partition identical, picks identical)."""
    U = torch.tensor(O.haar_unitary(784, 4001), device=DEV)
    occ = {p: fock_sample(U, list(range(28)), 24, generator=torch.Generator().manual_seed(44), indist=0.95,
                          precision=p) for p in ("f64", "mixed", "compensated")}
    assert (occ["f64"].sum(1) == 28).all()
    assert torch.equal(occ["f64"], occ["mixed"]) and torch.equal(occ["f64"], occ["compensated"])


def test_c5_shape_sampled_circuits_match_the_oracle():
    """Every 16th of the 256 small circuits of the many-instance configuration (seeded as the benchmark
    seeds them), 48 chains each with supplied uniforms: FP64 picks bit-exact against the oracle, both FP32
    forms' picks equal to FP64's, marginals within tolerance."""
    rng = np.random.default_rng(5000)
    spec = []
    for i in range(256):
        m = int(rng.choice([16, 24, 32, 48, 64]))
        n = int(rng.integers(4, min(12, m // 4) + 1))
        rng.uniform(0.6, 1.0)
        spec.append((m, n, 5000 + i))
    for m, n, seed in spec[::16]:
        U = O.haar_unitary(m, seed)
        r2 = np.random.default_rng(seed)
        S = 48
        sig = np.argsort(r2.random((S, n)), axis=1)
        u = r2.random((S, n))
        ref = O.chain(U[:, :n], np.zeros(S, np.int64), sig, u, marg=True)
        Ut = torch.tensor(U, device=DEV)
        f64 = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True)
        far = (ref["gap"] > 1e-11).all(axis=1)
        rows64 = f64["rows"].cpu().numpy()
        assert np.array_equal(rows64[far], ref["rows"][far]), (m, n)
        m64 = f64["marg"].cpu().numpy()
        for p in ("mixed", "compensated"):
            o = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, precision=p)
            assert np.array_equal(o["rows"].cpu().numpy(), rows64), (m, n, p)
            mp = o["marg"].cpu().numpy()
            for s in np.nonzero(far)[0]:
                for j in range(n):
                    assert _rel(m64[s, j], ref["marg"][s, j]) <= 1e-10
                    tol = 1e-8 if p == "compensated" else mixed_tol(j + 1)
                    assert _rel(mp[s, j], ref["marg"][s, j]) <= tol, (m, n, p, s, j)
