"""Parity of the CUDA path (through the C ABI) with the oracle and with the reference's recorded draws.

Tolerances: FP64 form — cofactors and marginals within 1e-10 relative (normwise) up to 24 columns,
growing 1.8x per column beyond (f64_tol), picks bit-exact;
mixed form — picks identical to the FP64 form's (the guard band sends ambiguous draws through the FP64
sweep), cofactors and marginals within the FP32 envelope mixed_tol(k) = 2e-7 * 1.35^k (about 1e-6 at
k = 10, 8e-5 at k = 20; the measured maxima sit 2-4x below it).  A pick is compared whenever the oracle's
draw lies farther than 1e-11 * total weight from every CDF step (closer draws are counted and must be
rare)."""
import functools
import math
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import oracle as O
from photonic_engines_b200 import _native as N
from photonic_engines_b200.clifford import fock_sample, laplace_cofactors_rows, sample_chains
from photonic_engines_b200.clifford.kernels import chain, pack_instances

pytestmark = pytest.mark.gpu
DEV = "cuda"
STEPS = np.load(os.path.join(GOLDEN, "steps.npz"))
CHAINS = np.load(os.path.join(GOLDEN, "chains.npz"))
LOSSLESS = sorted({k.split("__")[0] for k in CHAINS.files if k.endswith("__rows")})
IMPERFECT = sorted({k.split("__")[0] for k in CHAINS.files if k.endswith("__imperf")})
CONFIGS = [(32, 1), (64, 2), (128, 4), (256, 2), (256, 4), (128, 1)]
F64_TOL = 1e-10


def mixed_tol(k: int) -> float:
    """Relative error envelope of the mixed form at a step with k columns (k - 1 chosen rows)."""
    return 2e-7 * 1.35 ** k


def _rel(a, b):
    """Normwise relative difference; an all-zero reference compares absolutely."""
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / scale) if scale > 0 else float(np.abs(a).max())


# ------------------------------------------------------------------------------------------- cofactors

@pytest.mark.parametrize("block,tpl", CONFIGS)
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_cofactors_of_repeated_row_blocks_match_the_reference(block, tpl, precision):
    for i in range(len(STEPS["K1"])):
        K1 = int(STEPS["K1"][i])
        K = K1 + 1
        rows = STEPS["rows"][i, :K1]
        B = STEPS["blocks"][i, :K1, :K]
        m = int(rows.max()) + 1 if K1 else 1
        A = np.zeros((m, K), dtype=np.complex128)
        A[rows] = B
        P = laplace_cofactors_rows(torch.tensor(A[None], device=DEV), torch.tensor(rows[None], device=DEV),
                                   precision=precision, block_threads=block, tpl=tpl).cpu().numpy()[0]
        tol = 1e-12 if precision == "f64" else mixed_tol(K1)
        assert _rel(P, STEPS["P_ld"][i, :K]) <= tol, (i, precision, block, tpl)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_cofactors_structured_blocks(precision):
    """Zero columns (exact-zero products) and the all-ones block, per = (K - 1)! (check_cofactors.py:40-52)."""
    rng = np.random.default_rng(0)
    for K1 in (3, 6, 11):
        K = K1 + 1
        B = rng.normal(size=(4, K1, K)) + 1j * rng.normal(size=(4, K1, K))
        B[1][:, 0] = 0
        B[2][:, 0] = 0
        B[2][:, 2] = 0
        B[3][:, :] = 1
        rows = np.tile(np.arange(K1), (4, 1))
        P = laplace_cofactors_rows(torch.tensor(B, device=DEV), torch.tensor(rows, device=DEV),
                                   precision=precision).cpu().numpy()
        R = np.stack([O.ryser_cofactors(B[s]) if K1 <= 9 else O.cofactors(B[s], rows[s])[0] for s in range(4)])
        tol = 1e-11 if precision == "f64" else mixed_tol(K1)
        for s in (0, 1, 3):
            assert _rel(P[s], R[s]) <= tol
        assert np.abs(P[2]).max() == 0.0               # two zero columns: every cofactor is exactly zero
        assert abs(P[3, 0] - math.factorial(K1)) <= tol * math.factorial(K1)


@pytest.mark.parametrize("K1", [12, 16, 20, 23, 27, 31])
def test_cofactors_large_k_random_collisions(K1):
    """Random repeated-row blocks at large k (check_cuda.py:38-50) against the oracle."""
    rng = np.random.default_rng(K1)
    K, S, m = K1 + 1, 4, 2 * (K1 + 1)
    A = rng.normal(size=(S, m, K)) + 1j * rng.normal(size=(S, m, K))
    rows = rng.integers(0, m, size=(S, K1))
    if K1 >= 27:
        rows = rng.integers(0, 10, size=(S, K1))           # heavy collisions keep the oracle fast
    At, rt = torch.tensor(A, device=DEV), torch.tensor(rows, device=DEV)
    P64 = laplace_cofactors_rows(At, rt).cpu().numpy()
    Pmx = laplace_cofactors_rows(At, rt, precision="mixed").cpu().numpy()
    for s in range(S):
        ref, _ = O.cofactors(A[s][rows[s]], rows[s], precision="ld")
        assert _rel(P64[s], ref) <= 1e-10
        assert _rel(Pmx[s], ref) <= mixed_tol(K1)


# ------------------------------------------------------------------------------------------- golden chains

@pytest.mark.parametrize("name", LOSSLESS)
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_chains_reproduce_the_reference_draws(name, precision):
    U = torch.as_tensor(CHAINS[f"{name}__U"], device=DEV)
    in_modes = CHAINS[f"{name}__in_modes"].tolist()
    m, Bn, shots, gseed = CHAINS[f"{name}__meta"][:4].tolist()
    dp = torch.arange(Bn, device=DEV).repeat_interleave(shots)
    out = sample_chains(U, in_modes, CHAINS[f"{name}__sigma"], seeds=CHAINS[f"{name}__seeds"], dp=dp,
                        precision=precision)
    assert np.array_equal(out["rows"].cpu().numpy(), CHAINS[f"{name}__rows"])
    occ = fock_sample(U if Bn > 1 else U[0], in_modes, shots, generator=torch.Generator().manual_seed(gseed),
                      precision=precision)
    assert np.array_equal(occ.cpu().numpy(), CHAINS[f"{name}__occ"])


@pytest.mark.parametrize("name", IMPERFECT)
def test_loss_and_distinguishability_reproduce_the_reference_samples(name):
    U = torch.as_tensor(CHAINS[f"{name}__U"], device=DEV)
    in_modes = CHAINS[f"{name}__in_modes"].tolist()
    m, shots, gseed = CHAINS[f"{name}__meta"][:3].tolist()
    loss, indist = CHAINS[f"{name}__imperf"].tolist()
    occ = fock_sample(U, in_modes, shots, generator=torch.Generator().manual_seed(gseed),
                      loss=None if loss < 0 else loss, indist=None if indist < 0 else indist)
    assert np.array_equal(occ.cpu().numpy(), CHAINS[f"{name}__occ"])


# ------------------------------------------------------------------------------------------- oracle chains

def _random_chains(n, m, S, seed):
    U = O.haar_unitary(m, seed)
    rng = np.random.default_rng(seed)
    sig = np.argsort(rng.random((S, n)), axis=1)
    u = rng.random((S, n))
    return U, sig, u


@pytest.mark.parametrize("n,m,S,mode", [(6, 12, 64, "cta"), (6, 12, 64, "warp"), (12, 40, 32, "cta"),
                                        (12, 40, 32, "warp"), (16, 60, 24, "warp"), (20, 400, 24, "cta")])
def test_chains_match_the_oracle_with_supplied_uniforms(n, m, S, mode):
    U, sig, u = _random_chains(n, m, S, 1000 + n)
    ref = O.chain(U[:, :n], np.zeros(S, np.int64), sig, u, marg=True)
    Ut = torch.tensor(U, device=DEV)
    f64 = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, mode=mode)
    mix = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, precision="mixed", mode=mode)
    rows64 = f64["rows"].cpu().numpy()
    far = (ref["gap"] > 1e-11).all(axis=1)
    assert far.mean() > 0.9
    assert np.array_equal(rows64[far], ref["rows"][far])
    assert np.array_equal(mix["rows"].cpu().numpy(), rows64)
    m64, mmx = f64["marg"].cpu().numpy(), mix["marg"].cpu().numpy()
    for s in np.nonzero(far)[0]:
        for k in range(n):
            assert _rel(m64[s, k], ref["marg"][s, k]) <= F64_TOL
            assert _rel(mmx[s, k], ref["marg"][s, k]) <= mixed_tol(k + 1)


@pytest.mark.parametrize("n,m,S", [(10, 300, 48), (12, 900, 32), (6, 4200, 16)])
def test_warp_form_picks_over_many_modes_match_the_oracle(n, m, S):
    """The warp form's draw over more than 128 modes without the marginal output (the CDF kept at every
    128-mode piece, only the pick's piece formed again; past 4096 modes the whole CDF scanned twice): rows
    bit-exact against the oracle where its draws are far from a CDF step, the mixed form's picks equal."""
    U, sig, u = _random_chains(n, m, S, 2000 + m)
    ref = O.chain(U[:, :n], np.zeros(S, np.int64), sig, u, marg=False)
    Ut = torch.tensor(U, device=DEV)
    rows = sample_chains(Ut, list(range(n)), sig, uniforms=u, mode="warp")["rows"].cpu().numpy()
    mix = sample_chains(Ut, list(range(n)), sig, uniforms=u, mode="warp", precision="mixed")["rows"].cpu().numpy()
    far = (ref["gap"] > 1e-11).all(axis=1)
    assert far.mean() > 0.9
    assert np.array_equal(rows[far], ref["rows"][far])
    assert np.array_equal(mix, rows)


def f64_tol(k: int) -> float:
    """FP64 envelope at a step with k columns: 1e-10 up to 24, growing 1.8x per column beyond (sums of
    2^(k-2) terms; the FP64 oracle itself sits 1.9e-10 from its long-double form at k = 29)."""
    return F64_TOL * max(1.0, 1.8 ** (k - 24))


@functools.lru_cache(maxsize=None)
def _long_chain_case(n):
    """Three chains of n photons in m = 2n modes and the long-double oracle's rows, gaps and marginals."""
    m, S = 2 * n, 3
    U, sig, u = _random_chains(n, m, S, 500 + n)
    return U, sig, u, O.chain(U[:, :n], np.zeros(S, np.int64), sig, u, precision="ld", marg=True, threads=S)


@pytest.mark.parametrize("tpl", [0, 4])
@pytest.mark.parametrize("n", [22, 26, 29])
def test_long_chains_match_the_oracle_at_the_wide_tiers(n, tpl):
    """Chains of 22, 26 and 29 photons (the 24-, 28- and 32-column kernels) in the default two-thread
    lanes and in four-thread lanes, heavy steps split over the GPU, against the long-double oracle: FP64
    picks bit-exact and marginals within f64_tol(k); mixed picks equal to the FP64 picks, marginals within
    mixed_tol(k)."""
    U, sig, u, ref = _long_chain_case(n)
    Ut = torch.tensor(U, device=DEV)
    f64 = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, tpl=tpl, split=None)
    mix = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, tpl=tpl, split=None, precision="mixed")
    rows64 = f64["rows"].cpu().numpy()
    far = (ref["gap"] > 1e-11).all(axis=1)
    assert far.sum() >= 2
    assert np.array_equal(rows64[far], ref["rows"][far])
    assert np.array_equal(mix["rows"].cpu().numpy(), rows64)
    m64, mmx = f64["marg"].cpu().numpy(), mix["marg"].cpu().numpy()
    for s in np.nonzero(far)[0]:
        for k in range(n):
            assert _rel(m64[s, k], ref["marg"][s, k]) <= f64_tol(k + 1), (s, k)
            assert _rel(mmx[s, k], ref["marg"][s, k]) <= mixed_tol(k + 1), (s, k)


@pytest.mark.parametrize("block,tpl", CONFIGS)
def test_launch_shapes_give_identical_picks(block, tpl):
    n, m, S = 10, 30, 40
    U, sig, u = _random_chains(n, m, S, 77)
    ref = O.chain(U[:, :n], np.zeros(S, np.int64), sig, u)
    out = sample_chains(torch.tensor(U, device=DEV), list(range(n)), sig, uniforms=u, block_threads=block, tpl=tpl,
                        mode="cta")
    assert np.array_equal(out["rows"].cpu().numpy(), ref["rows"])


@pytest.mark.parametrize("tpl", [1, 2])
@pytest.mark.parametrize("n,m", [(3, 5), (9, 30), (14, 100)])
def test_warp_form_thread_groupings_give_identical_picks(tpl, n, m):
    S = 80
    U, sig, u = _random_chains(n, m, S, 55 + n)
    ref = O.chain(U[:, :n], np.zeros(S, np.int64), sig, u)
    for precision in ("f64", "mixed"):
        out = sample_chains(torch.tensor(U, device=DEV), list(range(n)), sig, uniforms=u, tpl=tpl, mode="warp",
                            precision=precision)
        assert np.array_equal(out["rows"].cpu().numpy(), ref["rows"])


# ------------------------------------------------------------------------------------------- distributions

@pytest.mark.parametrize("m,in_modes,shots", [(4, [0, 1, 2], 20000), (5, [0, 0, 1], 20000), (6, [0, 1, 2, 3], 30000)])
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_histogram_matches_the_exact_distribution(m, in_modes, shots, precision):
    U = O.haar_unitary(m, 100 + m)
    dist = O.exact_distribution(U, in_modes)
    occ = fock_sample(torch.tensor(U, device=DEV), in_modes, shots,
                      generator=torch.Generator(device=DEV).manual_seed(0), precision=precision)
    tvd, floor = O.tvd_and_floor(dist, occ.cpu().numpy())
    assert tvd < 2.5 * floor, (tvd, floor)


def test_lossy_histogram_matches_the_thinned_distribution():
    """Uniform loss eta on 3 photons: each photon survives independently, so the law is the mixture over
    surviving subsets of their exact distributions."""
    import itertools
    m, in_modes, eta, shots = 4, [0, 1, 2], 0.6, 40000
    U = O.haar_unitary(m, 5)
    dist: dict = {}
    for r in range(len(in_modes) + 1):
        for sub in itertools.combinations(range(len(in_modes)), r):
            w = eta ** r * (1 - eta) ** (len(in_modes) - r)
            part = O.exact_distribution(U, [in_modes[j] for j in sub]) if sub else {tuple([0] * m): 1.0}
            for k, p in part.items():
                dist[k] = dist.get(k, 0.0) + w * p
    occ = fock_sample(torch.tensor(U, device=DEV), in_modes, shots, loss=eta,
                      generator=torch.Generator(device=DEV).manual_seed(3))
    tvd, floor = O.tvd_and_floor(dist, occ.cpu().numpy())
    assert tvd < 2.5 * floor, (tvd, floor)


# ------------------------------------------------------------------------------------------- edge cases

def test_identity_and_hom():
    occ = fock_sample(torch.eye(3, dtype=torch.complex128, device=DEV), [0, 2, 2], 50,
                      generator=torch.Generator(device=DEV).manual_seed(0)).cpu().numpy()
    assert (occ == np.array([1, 0, 2])).all()
    hom = torch.tensor([[1, 1], [1, -1]], dtype=torch.complex128, device=DEV) / math.sqrt(2)
    occ = fock_sample(hom, [0, 1], 300, generator=torch.Generator(device=DEV).manual_seed(0)).cpu().numpy()
    assert not (occ == 1).all(1).any()


def test_batched_circuits_are_laid_out_as_b_times_shots():
    p0, p1 = [0, 1, 2, 3], [2, 3, 0, 1]
    U = torch.stack([torch.eye(4, dtype=torch.complex128)[p] for p in (p0, p1)]).to(DEV)
    occ = fock_sample(U, [0, 1], 8, generator=torch.Generator(device=DEV).manual_seed(0))
    assert occ[:8].tolist() == [[1, 1, 0, 0]] * 8
    assert occ[8:].tolist() == [[0, 0, 1, 1]] * 8
    occ = fock_sample(U, [0, 1], torch.tensor([3, 5]), generator=torch.Generator(device=DEV).manual_seed(0))
    assert occ.shape == (8, 4) and occ[:3].tolist() == [[1, 1, 0, 0]] * 3


def test_empty_requests_and_trivial_loss():
    U = torch.tensor(O.haar_unitary(5, 1), device=DEV)
    assert fock_sample(U, [0, 1], 0).shape == (0, 5)
    g = lambda: torch.Generator(device=DEV).manual_seed(4)
    assert torch.equal(fock_sample(U, [0, 1, 2], 16, generator=g(), loss=1.0), fock_sample(U, [0, 1, 2], 16, generator=g()))
    assert int(fock_sample(U, [0, 1, 2], 16, generator=g(), loss=0.0).sum()) == 0
    occ = fock_sample(U, [3], 100, generator=g())                    # one photon: K1 = 0 at every step
    assert (occ.sum(1) == 1).all()


def test_same_seed_same_samples_and_all_photons_placed():
    U = torch.tensor(O.haar_unitary(60, 9), device=DEV)
    a = fock_sample(U, list(range(14)), 200, generator=torch.Generator(device=DEV).manual_seed(5))
    b = fock_sample(U, list(range(14)), 200, generator=torch.Generator(device=DEV).manual_seed(5))
    c = fock_sample(U, list(range(14)), 200, generator=torch.Generator(device=DEV).manual_seed(6))
    assert torch.equal(a, b) and not torch.equal(a, c)
    assert (a.sum(1) == 14).all()


def test_an_out_of_range_column_is_reported_not_faulted():
    """The kernel's own bounds check turns a bad column index into a device status, read back as an error."""
    U = torch.tensor(O.haar_unitary(8, 1), device=DEV)
    acol, off, mm, nn = pack_instances(U, [0, 1, 2])
    cols = torch.tensor([[0, 1, 2], [0, 7, 1]], device=DEV)
    with pytest.raises(N.NativeError, match="device-side"):
        chain(acol, off, mm, nn, torch.zeros(2, dtype=torch.int64, device=DEV), cols, seeds=[1, 2, 3])
    rows, _, _ = chain(acol, off, mm, nn, torch.zeros(1, dtype=torch.int64, device=DEV), cols[:1], seeds=[1, 2, 3])
    assert rows.shape == (1, 3)


# ------------------------------------------------------------------------------------------- split steps

@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("k_split,nch", [(2, 1), (6, 3), (9, 16), (12, 64)])
def test_split_steps_match_single_cta_chains(precision, k_split, nch):
    """Heavy steps shared by nch CTAs per stream give the single-CTA chains (FP64 marginals within 1e-12)."""
    n, m, S = 14, 48, 6
    U, sig, u = _random_chains(n, m, S, 31)
    Ut = torch.tensor(U, device=DEV)
    a = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, precision=precision, split=False)
    b = sample_chains(Ut, list(range(n)), sig, uniforms=u, want_marg=True, precision=precision, split=(k_split, nch))
    assert torch.equal(a["rows"], b["rows"]) and torch.equal(a["occ"], b["occ"])
    ma, mb = a["marg"].cpu().numpy(), b["marg"].cpu().numpy()
    for s in range(S):
        for k in range(n):
            tol = 1e-12 if precision == "f64" else mixed_tol(k + 1)      # FP32 blocks start at other lanes
            assert _rel(mb[s, k], ma[s, k]) <= tol


@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("n,shapes", [(18, [(1, 128), (2, 256), (4, 256), (1, 64)]),
                                      (22, [(2, 128), (2, 64), (4, 256), (4, 128), (2, 128)])])
def test_split_steps_in_every_launch_shape_one_after_another(precision, n, shapes):
    """Split steps in launch shapes of variants compiled for 128- and 256-thread CTAs, in one process and
    in turn (an autotuner's order): each variant launches its own draw kernel, every shape gives the same
    picks."""
    m, S = 2 * n, 4
    U, sig, u = _random_chains(n, m, S, 71 + n)
    Ut = torch.tensor(U, device=DEV)
    first = None
    for tpl, block in shapes:
        out = sample_chains(Ut, list(range(n)), sig, uniforms=u, precision=precision, split=(12, 4), tpl=tpl,
                            block_threads=block)
        rows = out["rows"].cpu().numpy()
        first = rows if first is None else first
        assert np.array_equal(rows, first), (tpl, block)


def test_single_sample_uses_the_whole_gpu_and_matches_the_oracle():
    n, m = 18, 40
    U, sig, u = _random_chains(n, m, 1, 41)
    ref = O.chain(U[:, :n], np.zeros(1, np.int64), sig, u)
    out = sample_chains(torch.tensor(U, device=DEV), list(range(n)), sig, uniforms=u, split=None)
    assert np.array_equal(out["rows"].cpu().numpy(), ref["rows"])
    occ = fock_sample(torch.tensor(U, device=DEV), list(range(n)), 1, generator=torch.Generator(device=DEV).manual_seed(2))
    assert int(occ.sum()) == n


@pytest.mark.xfail(strict=True, reason="the plain mixed form's FP32 blocks err by ~2e-5 at 20 columns; the "
                                       "compensated form is the FP32 form within 1e-6")
def test_plain_mixed_form_meets_the_1e6_marginal_bound_at_n20():
    """Kept visible on purpose: the plain mixed form does NOT meet the north-star bound of 1e-6 at n = 20,
    m = 400 (measured 2e-5); its picks still equal FP64's (guard band).  Fails as expected."""
    n, m, S = 20, 400, 8
    U, sig, u = _random_chains(n, m, S, 4040)
    ref = O.chain(U[:, :n], np.zeros(S, np.int64), sig, u, precision="ld", marg=True, threads=S)
    mix = sample_chains(torch.tensor(U, device=DEV), list(range(n)), sig, uniforms=u, want_marg=True, precision="mixed")
    mm = mix["marg"].cpu().numpy()
    worst = max(_rel(mm[s, k], ref["marg"][s, k]) for s in range(S) for k in range(n))
    assert worst <= 1e-6, worst
