"""EmitterMPS inputs on the GPU (pe_emitter_weights through the C ABI): step weights against the reference's
recorded matrix_cofactor_weights and against the oracle's restatement at every kernel tier (k up to 18),
samples against the reference's recorded draws (same generator, same samples), the law against the exact
output distribution, and device-side index checks.  Tolerance: weights within 1e-10 relative (FP64)."""
import numpy as np
import pytest
import torch

from oracle import emitter_oracle as EO
from oracle import oracle as O
from photonic_engines_b200 import _native as N
from photonic_engines_b200.clifford import emitter_sample, sample
from photonic_engines_b200.clifford.emitter import _Terms, gap_terms, step_weights
from photonic_engines_b200.states import EmitterMPS
from test_emitter_cpu import CASES, case

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", CASES)
def test_step_weights_match_the_reference(name):
    st, U, steps, *_ = case(name)
    Ud = torch.as_tensor(U, device=DEV)
    terms = _Terms(st)
    for T, rows, fv, w in steps:
        k = len(T)
        fid = torch.tensor([0 if fv is None else int(np.argmax(np.abs(fv)))])
        rows_d = torch.zeros(1, st.n, dtype=torch.int64, device=DEV)
        rows_d[0, :k - 1] = torch.as_tensor(rows, dtype=torch.int64)
        got, nl = step_weights(Ud, st, torch.tensor([T]), rows_d, fid, terms, k)
        assert nl >= 1
        assert _rel(got[0].cpu().numpy(), w) < 1e-10, (name, T)


@pytest.mark.parametrize("name", CASES)
def test_samples_are_the_reference_samples(name):
    st, U, _, shots, seed, occ = case(name)
    got = emitter_sample(st, torch.as_tensor(U, device=DEV), shots, generator=torch.Generator().manual_seed(seed))
    assert got.device.type == "cuda"
    assert (got.cpu().numpy() == occ).all()
    got2 = sample(st, torch.as_tensor(U, device=DEV), shots, generator=torch.Generator().manual_seed(seed))
    assert torch.equal(got, got2)


def _random_emitter(n, L, seed, final=True):
    rng = np.random.default_rng(seed)
    ops = rng.normal(size=(n, L, 2, 2)) + 1j * rng.normal(size=(n, L, 2, 2))
    f = (rng.normal(size=2) + 1j * rng.normal(size=2)) if final else None
    return EmitterMPS(ops=ops, modes=tuple(tuple(range(k * L, (k + 1) * L)) for k in range(n)),
                      s0=rng.normal(size=2) + 1j * rng.normal(size=2), m=n * L + 3, final=f), rng


@pytest.mark.parametrize(("n", "L", "ks", "final"), [(10, 2, (6, 8), True), (14, 1, (11, 14), False),
                                                    (14, 2, (12, 16 - 2), True), (20, 1, (17, 18), True),
                                                    (20, 2, (17,), False)])
def test_every_tier_matches_the_oracle(n, L, ks, final):
    """Several streams with different placed slots, rows and final spins in one launch, at each k."""
    st, rng = _random_emitter(n, L, 100 + n + L, final)
    U = O.haar_unitary(st.m, 7 + n)
    Ud = torch.as_tensor(U, device=DEV)
    terms = _Terms(st)
    S = 3
    for k in ks:
        T = torch.tensor([sorted(rng.choice(n, size=k, replace=False).tolist()) for _ in range(S)])
        rows = torch.as_tensor(rng.integers(0, st.m, size=(S, n)), dtype=torch.int64)
        fid = torch.as_tensor(rng.integers(0, 1 if final else 2, size=S))
        got, _ = step_weights(Ud, st, T, rows.to(DEV), fid, terms, k)
        got = got.cpu().numpy()
        for s in range(S):
            fv = None if final else torch.eye(2, dtype=torch.complex128)[int(fid[s])]
            kept, s0, mats, f = gap_terms(st, T[s].tolist(), fv)
            colmode = np.array([list(st.modes[j]) for j in kept])
            want = EO.matrix_weights(U, colmode, rows[s, :k - 1].tolist(), s0.numpy(), mats.numpy(), f.numpy())
            assert _rel(got[s], want) < 1e-10, (n, L, k, s)


def test_samples_follow_the_exact_distribution():
    """A traced emitter, 3 photons in 9 modes: histogram of 20 000 samples against the exact law."""
    st, _ = _random_emitter(3, 2, 41, final=False)
    U = O.haar_unitary(st.m, 41)
    dist = EO.exact_distribution(U, st.ops, st.modes, st.s0, None)
    occ = emitter_sample(st, torch.as_tensor(U, device=DEV), 20000, generator=torch.Generator().manual_seed(3))
    tvd, floor = O.tvd_and_floor(dist, occ.cpu().numpy())
    assert tvd < 2.5 * floor, (tvd, floor)


def test_an_out_of_range_mode_is_reported_not_faulted():
    L = N.load()
    m, k = 6, 2
    ut = torch.zeros(m, m, 2, dtype=torch.float64, device=DEV)
    rows = torch.zeros(1, 1, dtype=torch.int64, device=DEV)
    colmode = torch.tensor([[[0], [m + 5]]], dtype=torch.int32, device=DEV)                 # mode beyond U
    s0 = torch.zeros(1, 2, 2, dtype=torch.float64, device=DEV)
    mats = torch.zeros(1, k, 1, 2, 2, 2, dtype=torch.float64, device=DEV)
    lane = torch.zeros(1, dtype=torch.int64, device=DEV)
    nlan = torch.ones(1, dtype=torch.int64, device=DEV)
    amp = torch.zeros(1, m, 2, dtype=torch.float64, device=DEV)
    w = torch.zeros(1, m, dtype=torch.float64, device=DEV)
    ws = torch.zeros(256, dtype=torch.uint8, device=DEV)
    rc = L.pe_emitter_weights(ut.data_ptr(), m, m, rows.data_ptr(), 1, colmode.data_ptr(), 1, k, 1, 2, s0.data_ptr(),
                              s0.data_ptr(), mats.data_ptr(), 1, lane.data_ptr(), lane.data_ptr(), lane.data_ptr(),
                              nlan.data_ptr(), 1, amp.data_ptr(), w.data_ptr(), ws.data_ptr(), 256,
                              N.stream_handle(torch.device(DEV)))
    assert rc == 0
    st, _ = N.read_status(ws)
    assert st == N.PE_ERR_DEVICE
    assert L.pe_emitter_weights(ut.data_ptr(), m, m, rows.data_ptr(), 1, colmode.data_ptr(), 1, k, 1, 3,
                                s0.data_ptr(), s0.data_ptr(), mats.data_ptr(), 1, lane.data_ptr(), lane.data_ptr(),
                                lane.data_ptr(), nlan.data_ptr(), 1, amp.data_ptr(), w.data_ptr(), ws.data_ptr(), 256,
                                N.stream_handle(torch.device(DEV))) == N.PE_ERR_SIZE            # chi = 3


@pytest.mark.parametrize(("n", "L", "ks", "final"), [(10, 2, (1, 2, 6, 8), True), (12, 1, (9, 12), False),
                                                    (14, 2, (12,), True), (20, 1, (17, 18), False)])
def test_fused_steps_match_the_oracle(n, L, ks, final):
    """pe_emitter_count + pe_emitter_step (terms assembled on the device from the per-state tables)."""
    from photonic_engines_b200.clifford.emitter import fused_step_weights, tables_for
    st, rng = _random_emitter(n, L, 300 + n + L, final)
    U = O.haar_unitary(st.m, 9 + n)
    Ud = torch.as_tensor(U, device=DEV)
    ut = torch.view_as_real(Ud.transpose(0, 1).contiguous()).contiguous()
    tb = tables_for(st, DEV)
    S = 4
    for k in ks:
        T = torch.tensor([sorted(rng.choice(n, size=k, replace=False).tolist()) for _ in range(S)], dtype=torch.int32)
        rows = torch.as_tensor(rng.integers(0, st.m, size=(S, n)), dtype=torch.int64)
        fid = torch.as_tensor(rng.integers(0, 1 if final else 2, size=S), dtype=torch.int32)
        ws = torch.zeros(256, dtype=torch.uint8, device=DEV)
        got, _ = fused_step_weights(ut, st.m, st, T.to(DEV), rows.to(DEV), fid.to(DEV), tb, ws)
        assert N.read_status(ws)[0] == 0
        got = got.cpu().numpy()
        for s in range(S):
            fv = None if final else torch.eye(2, dtype=torch.complex128)[int(fid[s])]
            kept, s0, mats, f = gap_terms(st, T[s].tolist(), fv)
            colmode = np.array([list(st.modes[j]) for j in kept])
            want = EO.matrix_weights(U, colmode, rows[s, :k - 1].tolist(), s0.numpy(), mats.numpy(), f.numpy())
            assert _rel(got[s], want) < 1e-10, (n, L, k, s)


# ------------------------------------------------------------------------------------------- loss / indist
from test_emitter_cpu import IMP, IMP_CASES  # noqa: E402


@pytest.mark.parametrize("c", IMP_CASES)
def test_imperfect_emitter_samples_reproduce_the_reference(c):
    """Loss and x-model partial distinguishability (lost labels unravelled or traced, lone photons' rows,
    chains over the interfering slots grouped by count): a seeded CPU generator gives the occupations the
    reference's emitter_sample recorded."""
    st, *_ = case(str(IMP[f"{c}__name"]))
    U = torch.as_tensor(IMP[f"{c}__U"], device=DEV)
    eta, x, unravel = IMP[f"{c}__imperf"].tolist()
    shots, seed = (int(v) for v in IMP[f"{c}__shots_seed"])
    occ = emitter_sample(st, U, shots, generator=torch.Generator().manual_seed(seed),
                         loss=None if eta < 0 else eta, indist=None if x < 0 else x, unravel=bool(unravel))
    assert np.array_equal(occ.cpu().numpy(), IMP[f"{c}__occ"])


def test_lossy_emitter_law_matches_the_exact_mixture():
    """A lossy traced emitter (n = 4, 2 labels): the sampled law against the exact mixture over the
    surviving photons' reduced states (oracle: each survivor subset weighted eta^|T| (1 - eta)^(n - |T|),
    the explicit reduced density matrix of T and Ryser permanents)."""
    st, U, *_ = case("rand_n4_L2_t")
    eta, shots = 0.6, 30000
    dist = EO.lossy_distribution(U, st.ops, st.modes, st.s0, st.final, eta)
    assert abs(sum(dist.values()) - 1.0) < 1e-9
    occ = emitter_sample(st, torch.as_tensor(U, device=DEV), shots, generator=torch.Generator().manual_seed(3),
                         loss=eta)
    tvd, floor = O.tvd_and_floor(dist, occ.cpu().numpy())
    assert tvd < 2.5 * floor, (tvd, floor)
