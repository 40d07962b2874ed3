"""Host-side logic of `fock_sample` on the CPU: the chain plan (sigma / seed draws, loss and partial
distinguishability partition, grouping, singleton routing) must consume a seeded generator exactly as the
reference does.  The oracle plays the chains of the plan, and the assembled occupations must equal the
ones the reference's own `fock_sample` returned (tests/golden/chains.npz)."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import oracle as O
from photonic_engines_b200.clifford.sampler import assemble_occupations, plan_chains

CHAINS = np.load(os.path.join(GOLDEN, "chains.npz"))
LOSSLESS = sorted({k.split("__")[0] for k in CHAINS.files if k.endswith("__rows")})
IMPERFECT = sorted({k.split("__")[0] for k in CHAINS.files if k.endswith("__imperf")})


def _play(plan, U, in_modes):
    """Run every chain of the plan on the oracle (grouped by photon count), then assemble occupations."""
    A = U[:, :, in_modes].numpy()
    rows = np.zeros((plan.C, plan.n), dtype=np.int64)
    nk = np.full(plan.C, plan.n) if plan.nk is None else plan.nk.numpy()
    for k in sorted(set(nk.tolist())):
        sel = np.nonzero(nk == k)[0]
        u = O.chain_uniforms(plan.seeds.numpy(), plan.seed_row.numpy()[sel], plan.rng_off.numpy()[sel], k)
        out = O.chain(A, plan.dp.numpy()[sel], plan.cols.numpy()[sel, :k], u)
        rows[sel, :k] = out["rows"]
    return assemble_occupations(plan, torch.as_tensor(rows), U.shape[-1]).numpy()


@pytest.mark.parametrize("name", LOSSLESS)
def test_lossless_plan_reproduces_the_reference_samples(name):
    U = torch.as_tensor(CHAINS[f"{name}__U"])
    in_modes = CHAINS[f"{name}__in_modes"].tolist()
    m, Bn, shots, gseed = CHAINS[f"{name}__meta"][:4].tolist()
    S = Bn * shots
    dp_all = torch.arange(Bn).repeat_interleave(shots)
    plan = plan_chains(U, in_modes, S, dp_all, torch.Generator().manual_seed(gseed), None, None, 1 << 18)
    assert torch.equal(plan.cols, torch.as_tensor(CHAINS[f"{name}__sigma"]))
    assert torch.equal(plan.seeds[0], torch.as_tensor(CHAINS[f"{name}__seeds"]))
    assert np.array_equal(_play(plan, U, in_modes), CHAINS[f"{name}__occ"])


def test_max_streams_splits_a_pass_into_chunks_with_their_own_draws():
    U = torch.as_tensor(O.haar_unitary(6, 2))[None]
    plan = plan_chains(U, [0, 1, 2], 10, torch.zeros(10, dtype=torch.int64), torch.Generator().manual_seed(1),
                       None, None, 4)
    assert plan.seeds.shape == (3, 3)
    assert plan.seed_row.tolist() == [0] * 4 + [1] * 4 + [2] * 2
    assert plan.rng_off.tolist() == [0, 1, 2, 3, 0, 1, 2, 3, 0, 1]


@pytest.mark.parametrize("name", IMPERFECT)
def test_imperfect_plan_reproduces_the_reference_samples(name):
    U = torch.as_tensor(CHAINS[f"{name}__U"])
    in_modes = CHAINS[f"{name}__in_modes"].tolist()
    m, shots, gseed = CHAINS[f"{name}__meta"][:3].tolist()
    loss, indist = CHAINS[f"{name}__imperf"].tolist()
    loss = None if loss < 0 else loss
    indist = None if indist < 0 else indist
    plan = plan_chains(U[None], in_modes, shots, torch.zeros(shots, dtype=torch.int64),
                       torch.Generator().manual_seed(gseed), loss, indist, 1 << 18)
    occ = _play(plan, U[None], in_modes)
    assert np.array_equal(occ, CHAINS[f"{name}__occ"])
    assert (occ.sum(1) <= len(in_modes)).all()


def test_loss_zero_transmission_returns_empty_samples():
    U = torch.as_tensor(O.haar_unitary(5, 3))[None]
    plan = plan_chains(U, [0, 1, 2], 8, torch.zeros(8, dtype=torch.int64), torch.Generator().manual_seed(0), 0.0,
                       None, 1 << 18)
    assert plan.C == 0 and plan.single_ids is None
    assert assemble_occupations(plan, None, 5).sum() == 0


@pytest.mark.parametrize(("n", "m", "S", "eta", "in_modes", "B"), [
    (20, 40, 1024, 0.5, list(range(20)), 1), (20, 40, 1024, 0.9, list(range(20)), 1),
    (8, 12, 500, 0.3, [0, 2, 4, 6, 8, 9, 10, 11], 2), (6, 9, 300, 0.2, [5, 1, 3, 0, 8, 2], 1),
    (32, 64, 200, 0.8, list(range(32)), 1)])
def test_loss_only_plan_in_tensor_ops_is_the_general_plan(n, m, S, eta, in_modes, B):
    """The vectorised plan for uniform loss (distinct input modes) makes the same draws and the same passes,
    chains, order and classical routings as the reference-ordered loop over role groups."""
    import torch
    from oracle.oracle import haar_unitary
    from photonic_engines_b200.clifford.sampler import plan_chains
    U = torch.stack([torch.as_tensor(haar_unitary(m, 3 + b)) for b in range(B)])
    dp = torch.arange(B).repeat_interleave(S // B)
    a = plan_chains(U, in_modes, dp.shape[0], dp, torch.Generator().manual_seed(7), eta, None, 128)
    b = plan_chains(U, in_modes, dp.shape[0], dp, torch.Generator().manual_seed(7), eta, None, 128, _force_general=True)
    assert a.passes == b.passes and a.C == b.C
    for f in ("dp", "cols", "nk", "seeds", "seed_row", "rng_off", "out_row", "order", "single_ids", "single_rows"):
        x, y = getattr(a, f), getattr(b, f)
        assert (x is None and y is None) or torch.equal(x, y), f


@pytest.mark.parametrize(("heavy", "n", "slots", "expect"), [
    (200, 28, 296, (17, 64)),       # 200 streams of 28 photons: 24 waves of the resident CTAs
    (2000, 20, 296, None),          # many streams: one CTA each already fills the GPU
    (1, 20, 296, (17, 64)),         # one stream: as many CTAs as the cap (2^18 terms / 32 lanes) allows
    (3, 6, 296, None),              # short chains are never split
])
def test_split_plan_sizes_the_ctas_per_stream_from_the_resident_slots(monkeypatch, heavy, n, slots, expect):
    """The split planner on the CPU, with the resident-CTA count the library would report stubbed: nch is a
    power of two filling SPLIT_FILL (SPLIT_FILL_LONG from 24 photons) waves, capped; k_split leaves every
    split step several Gray lanes per CTA."""
    from photonic_engines_b200.clifford import kernels as K
    monkeypatch.setattr(K, "_split_slots", lambda *a: slots)
    plan = K.split_plan(heavy, n, "cuda:0", 128, 1, "f64")
    if expect is None:
        assert plan is None
        return
    k, nch = plan
    assert nch & (nch - 1) == 0 and nch <= K.NCH_MAX
    waves = K.SPLIT_FILL_LONG if n >= 24 else K.SPLIT_FILL
    assert heavy * nch >= waves * slots or nch == min(K.NCH_MAX, (1 << (n - 2)) // (32 * 128))
    assert (1 << (k - 2)) >= 4 * nch * 128 and (1 << (k - 3)) < 4 * nch * 128
    assert (k, nch) == expect


def test_tier_plan_cuts_the_longest_first_queue(monkeypatch):
    """Length tiers of a ragged call on the CPU (resident split CTAs stubbed): consecutive queue ranges,
    longest first; the few chains above 24 photons split, a crowd of them not; the last tier in the warp form
    only when its streams fill the GPU's warps."""
    from photonic_engines_b200.clifford import kernels as K
    monkeypatch.setattr(K, "_split_slots", lambda *a: 296)
    monkeypatch.setattr(K, "use_warp_form", lambda S, n, d: n <= 12 or S >= 64 * 148)
    t = K.tier_plan({27: 3, 25: 2, 22: 40, 18: 500, 15: 3000, 9: 100}, 30, "f64", "cuda:0")
    assert [(a, b, k, mode) for a, b, k, mode, _ in t] == [(0, 5, 27, 2), (5, 45, 22, 0), (45, 545, 18, 0),
                                                          (545, 3645, 15, 0)]
    assert t[0][4] is not None
    t = K.tier_plan({27: 5000, 22: 10}, 30, "f64", "cuda:0")
    assert t[0][3] == 0 and t[0][4] is None                     # enough long chains to fill the GPU whole
    t = K.tier_plan({12: 100, 7: 50}, 12, "f64", "cuda:0")
    assert t == [(0, 150, 12, 1, None)]                          # one tier: the plain launch runs it
    assert K.tier_plan({}, 30, "f64", "cuda:0") == []
