"""The batched sampler (many circuits, device-side loss / distinguishability partition, one persistent
launch, CUDA-graph replay): exact law at small sizes, per-circuit layout, graph replays."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from photonic_engines_b200.clifford import BatchedSampler

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.mark.parametrize("precision", ["f64", "mixed", "compensated"])
@pytest.mark.parametrize("eta,x", [(0.7, 1.0), (1.0, 0.6), (0.8, 0.7)])
def test_batched_law_matches_the_exact_imperfect_distribution(precision, eta, x):
    m, in_modes, shots = 4, [0, 1, 2], 40000
    U = O.haar_unitary(m, 8)
    dist = O.imperfect_distribution(U, in_modes, eta, x)
    assert abs(sum(dist.values()) - 1) < 1e-9
    bs = BatchedSampler([(torch.tensor(U, device=DEV), in_modes)], shots, loss=eta, indist=x, precision=precision,
                        seed=5, tune=False)
    occ = bs.sample().clone()
    bs.check()
    tvd, floor = O.tvd_and_floor(dist, occ.cpu().numpy())
    assert tvd < 2.5 * floor, (tvd, floor)


def test_many_circuits_of_different_sizes_keep_their_rows():
    """Permutation circuits of different m and n: lossless shots land deterministically, per circuit."""
    rng = np.random.default_rng(0)
    circuits, expect = [], []
    for g in range(12):
        m = int(rng.choice([8, 16, 24, 48]))
        n = int(rng.integers(2, min(8, m // 2) + 1))
        perm = rng.permutation(m)
        U = torch.eye(m, dtype=torch.complex128)[perm].to(DEV)       # U[perm[i], i] = 1
        modes = list(range(n))
        occ = np.zeros(m, dtype=np.int64)
        for j in modes:
            occ[np.nonzero(perm == j)[0][0]] += 1
        circuits.append((U, modes))
        expect.append(occ)
    bs = BatchedSampler(circuits, 50, precision="mixed", seed=1, tune=False)
    occ = bs.sample().cpu().numpy()
    bs.check()
    for g, e in enumerate(expect):
        rows = occ[bs.rows_of(g)]
        assert (rows[:, : len(e)] == e).all()
        assert (rows[:, len(e):] == 0).all()


def test_graph_replays_draw_fresh_samples_and_conserve_photons():
    U = torch.tensor(O.haar_unitary(24, 3), device=DEV)
    circuits = [(U, list(range(10))), (U[:16, :16].clone(), list(range(5)))]
    bs = BatchedSampler(circuits, 500, loss=[0.6, 0.9], precision="f64", seed=2, tune=True)
    a = bs.sample().clone()
    b = bs.sample().clone()
    bs.check()
    assert not torch.equal(a, b)
    for occ in (a, b):
        assert int(occ[bs.rows_of(0)].sum(1).max()) <= 10 and int(occ[bs.rows_of(1)].sum(1).max()) <= 5
    mean_kept = a[bs.rows_of(0)].sum(1).double().mean().item()
    assert abs(mean_kept - 6.0) < 5 * math.sqrt(10 * 0.6 * 0.4 / 500)


def test_graph_and_eager_paths_agree_in_law():
    U = O.haar_unitary(5, 4)
    circ = [(torch.tensor(U, device=DEV), [0, 1])]
    dist = O.imperfect_distribution(U, [0, 1], 0.9, 0.8)
    for graph in (True, False):
        bs = BatchedSampler(circ, 30000, loss=0.9, indist=0.8, seed=11, graph=graph, tune=False)
        tvd, floor = O.tvd_and_floor(dist, bs.sample().cpu().numpy())
        assert tvd < 2.5 * floor


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_length_tiers_give_the_single_launch_samples(precision):
    """Lossy, partially distinguishable chains of up to 24 photons: the tiered launches (> 20, 17..20 and
    <= 16 photons, the last in the warp form, on three streams) draw the samples of one launch sized to
    the longest chain (same generator, same partition, same picks)."""
    U = torch.tensor(O.haar_unitary(48, 8), device=DEV)
    circ = [(U, list(range(24)))]
    out = []
    for tiers in (True, False):
        bs = BatchedSampler(circ, 3000, loss=0.7, indist=0.9, precision=precision, seed=5, tune=False, tiers=tiers)
        assert bool(bs.tiers) == tiers
        out.append((bs.sample().clone(), bs.sample().clone()))
        bs.check()
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_long_chain_split_tier_gives_the_single_launch_samples(precision):
    """Chains of 25 and 26 photons (a 26-photon circuit at eta = 0.78, 1 600 shots: about a dozen per batch)
    run in their own tier with their heavy steps split over many CTAs (pe_fock_chain_range_split); the
    samples equal those of one launch sized to the longest chain, which runs every chain in one CTA."""
    U = torch.tensor(O.haar_unitary(60, 26), device=DEV)
    circ = [(U, list(range(26)))]
    out = []
    for tiers in (True, False):
        bs = BatchedSampler(circ, 1600, loss=0.78, precision=precision, seed=9, tune=False, tiers=tiers)
        if tiers:
            assert bs.long_split is not None and bs.tiers[0][1] == 2
            assert int((bs.nk > 24).sum()) >= 0
        out.append((bs.sample().clone(), bs.sample().clone()))
        bs.check()
    n_long = int((bs.nk > 24).sum())
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1]), n_long


def test_a_tier_reports_a_chain_longer_than_its_kernel_and_a_bad_range():
    from photonic_engines_b200 import _native as N
    from photonic_engines_b200.clifford.kernels import pack_instances
    L = N.load()
    U = torch.tensor(O.haar_unitary(40, 2), device=DEV)
    n, S = 20, 4
    acol, off, mm, nn = pack_instances(U, list(range(n)))
    a2 = torch.view_as_real(acol.contiguous()) if acol.dtype != torch.float64 else acol
    dp = torch.zeros(S, dtype=torch.int64, device=DEV)
    cols = torch.arange(n, device=DEV).repeat(S, 1).contiguous()
    nk = torch.tensor([18, 12, 10, 5], dtype=torch.int32, device=DEV)
    order = torch.arange(S, device=DEV)
    seeds = torch.arange(1, n + 1, device=DEV)[None].contiguous()
    rows = torch.zeros(S, n, dtype=torch.int64, device=DEV)
    for qr, nk_max in (([0, S], 16), ([3, 1], 20)):
        qrange = torch.tensor(qr, dtype=torch.int64, device=DEV)
        ws = N.workspace(torch.device(DEV))
        rc = L.pe_fock_chain_range(0, N.ptr(a2), N.ptr(off), N.ptr(mm), N.ptr(nn), 1, 40, S, N.ptr(dp), N.ptr(nk),
                                   N.ptr(cols), n, None, N.ptr(seeds), None, None, N.ptr(order), N.ptr(rows), None,
                                   40, None, 40, N.ptr(ws), ws.numel(), 0, 0, 0, N.ptr(qrange), nk_max,
                                   1 if nk_max <= 16 else 0, N.stream_handle(torch.device(DEV)))
        assert rc == 0
        assert N.read_status(ws)[0] == N.PE_ERR_DEVICE, (qr, nk_max)
