"""EmitterMPS inputs on the host: the oracle pinned on the reference's own outputs (tests/golden/emitter.npz:
step weights of emitter_reference.matrix_cofactor_weights and occupations drawn by emitter_sampler.
sample_torch), the pure-term decomposition of the reduced state, and argument checks.  The reference's
tests this follows: tests/clifford/test_emitter_reference.py:88-126, test_emitter_sampler.py:58-72."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import emitter_oracle as EO
from photonic_engines_b200.clifford import emitter_sample
from photonic_engines_b200.clifford.emitter import final_spin_distribution, gap_terms
from photonic_engines_b200.states import EmitterMPS

EMIT = np.load(os.path.join(GOLDEN, "emitter.npz"))
CASES = sorted({k.split("__")[0] for k in EMIT.files})
FAST = [c for c in CASES if c not in ("caterpillar_n5", "rand_n5_L2_f")]      # oracle sampler under ~2 s


def case(name):
    z = {k.split("__")[1]: EMIT[k] for k in EMIT.files if k.startswith(name + "__")}
    fin = z["final"]
    st = EmitterMPS(ops=z["ops"], modes=tuple(tuple(int(x) for x in r) for r in z["modes"]), s0=z["s0"],
                    m=int(z["m"][0]), final=fin if fin.size else None)
    steps = []
    for i in range(z["step_T"].shape[0]):
        T = [int(t) for t in z["step_T"][i] if t >= 0]
        rows = [int(r) for r in z["step_rows"][i] if r >= 0]
        fv = None if st.final is not None else np.eye(2)[int(z["step_final"][i])]
        steps.append((T, rows, fv, z["step_w"][i]))
    return st, z["U"], steps, int(z["shots_seed"][0]), int(z["shots_seed"][1]), z["occ"]


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", CASES)
def test_density_oracle_reproduces_the_reference_step_weights(name):
    st, U, steps, *_ = case(name)
    for T, rows, fv, w in steps:
        f = st.final if fv is None else fv
        assert _rel(EO.candidate_weights(U, st.ops, st.modes, st.s0, f, T, rows), w) < 1e-12


@pytest.mark.parametrize("name", FAST)
def test_oracle_sampler_reproduces_the_reference_draws(name):
    st, U, _, shots, seed, occ = case(name)
    got = EO.sample(U, st.ops, st.modes, st.s0, st.final, shots, torch.Generator().manual_seed(seed))
    assert (got == occ).all()


@pytest.mark.parametrize("name", CASES)
def test_pure_terms_give_the_reference_weights(name):
    """The host decomposition into pure terms, summed by the oracle's matrix-cofactor restatement."""
    st, U, steps, *_ = case(name)
    for T, rows, fv, w in steps:
        kept, s0, mats, f = gap_terms(st, T, None if fv is None else torch.as_tensor(fv, dtype=torch.complex128))
        colmode = np.array([list(st.modes[j]) for j in kept])
        assert _rel(EO.matrix_weights(U, colmode, rows, s0.numpy(), mats.numpy(), f.numpy()), w) < 1e-12


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_pure_terms_reconstruct_the_reduced_density(seed):
    """sum_e |psi_e><psi_e| = rho_T of the placed photons (emitter_reference.gap_kraus_terms' contract)."""
    rng = np.random.default_rng(seed)
    n, L = 6, 2
    ops = rng.normal(size=(n, L, 2, 2)) + 1j * rng.normal(size=(n, L, 2, 2))
    st = EmitterMPS(ops=ops, modes=tuple(tuple(range(2 * k, 2 * k + 2)) for k in range(n)),
                    s0=rng.normal(size=2) + 1j * rng.normal(size=2), m=2 * n,
                    final=rng.normal(size=2) + 1j * rng.normal(size=2))
    c = np.einsum("...s,s->...", EO.coefficient_tensor(st.ops, st.s0), np.conj(st.final))
    for T in ([0, 3], [1, 2, 5], [4], [0, 2, 4, 5], list(range(6))):
        kept, s0, mats, f = gap_terms(st, T)
        rho = np.zeros((L ** len(T), L ** len(T)), dtype=np.complex128)
        for e in range(s0.shape[0]):
            psi = np.zeros([L] * len(T), dtype=np.complex128)
            for x in np.ndindex(*psi.shape):
                v = s0[e].numpy()
                for j, xj in enumerate(x):
                    v = mats[e, j, xj].numpy() @ v
                psi[x] = np.conj(f[e].numpy()) @ v
            psi = psi.reshape(-1)
            rho += np.outer(psi, psi.conj())
        want = EO.reduced_density(c, kept)
        assert np.abs(rho - want).max() < 1e-10 * np.abs(want).max(), T


def test_final_spin_distribution_matches_the_coefficient_tensor():
    st, *_ = case("rand_n4_L2_t")
    p = final_spin_distribution(st).numpy()
    assert np.allclose(p, EO.final_distribution(st.ops, st.s0), rtol=1e-12)


def test_emitter_state_checks():
    ops = np.zeros((2, 2, 2, 2), dtype=np.complex128)
    with pytest.raises(ValueError):
        EmitterMPS(ops=ops, modes=((0, 1), (1, 2)), s0=[1, 0], m=4)             # a mode used twice
    with pytest.raises(ValueError):
        EmitterMPS(ops=ops, modes=((0, 1), (2, 3)), s0=[1, 0, 0], m=4)          # s0 of the wrong size
    with pytest.raises(ValueError):
        EmitterMPS(ops=ops, modes=((0, 1), (2, 5)), s0=[1, 0], m=4)             # mode out of range


def test_emitter_sample_argument_checks():
    st, U, *_ = case("rand_n3_L2_f")
    U = torch.as_tensor(U)
    from photonic_engines_b200.imperfections import Distinguishability
    with pytest.raises(NotImplementedError):                       # several interfering species
        emitter_sample(st, U, 4, indist=Distinguishability(species=(0.5, 0.3)))
    with pytest.raises(ValueError):
        emitter_sample(st, U, 4, loss=1.5)
    with pytest.raises(NotImplementedError):
        emitter_sample(EmitterMPS(ops=np.zeros((2, 1, 3, 3)), modes=((0,), (1,)), s0=[1, 0, 0], m=3), U[:3, :3], 2)
    with pytest.raises(ValueError):
        emitter_sample(st, U, 4, backend="nope")


@pytest.mark.parametrize("final", [True, False])
def test_batched_lanes_are_the_per_set_terms(final):
    """The per-state tables assemble, for many placed-photon sets at once, exactly gap_terms' terms
    (same lanes, same order, same values)."""
    from photonic_engines_b200.clifford.emitter import _Tables
    rng = np.random.default_rng(3 + final)
    n = 7
    ops = rng.normal(size=(n, 2, 2, 2)) + 1j * rng.normal(size=(n, 2, 2, 2))
    st = EmitterMPS(ops=ops, modes=tuple(tuple(range(2 * k, 2 * k + 2)) for k in range(n)), s0=rng.normal(size=2),
                    m=15, final=(rng.normal(size=2) + 1j * rng.normal(size=2)) if final else None)
    tb = _Tables(st, "cpu")
    for k in range(1, n + 1):
        T = torch.tensor([sorted(rng.choice(n, size=k, replace=False).tolist()) for _ in range(6)])
        fid = torch.as_tensor(rng.integers(0, 1 if final else 2, size=6))
        s0, mats, f, lstart, nlan = tb.lanes(T, fid)
        for s in range(6):
            fv = None if final else torch.eye(2, dtype=torch.complex128)[int(fid[s])]
            _, a0, am, af = gap_terms(st, T[s].tolist(), fv)
            sl = slice(int(lstart[s]), int(lstart[s] + nlan[s]))
            assert torch.equal(a0, s0[sl]) and torch.equal(am, mats[sl]) and torch.equal(af, f[sl]), (k, s)


IMP = np.load(os.path.join(GOLDEN, "emitter_imperfect.npz"))
IMP_CASES = sorted({k.split("__")[0] for k in IMP.files})


@pytest.mark.parametrize("c", IMP_CASES)
def test_slot_outcomes_reproduce_the_reference_draws(c):
    """Lost labels, lone photons' rows and the final spin drawn slot by slot (the reference's
    emitter_terms.sample_slot_outcomes on recorded fates, seeded CPU generator): the same values."""
    from photonic_engines_b200.clifford.emitter import slot_outcomes
    st, *_ = case(str(IMP[f"{c}__name"]))
    U = torch.as_tensor(IMP[f"{c}__U"])
    fates = torch.as_tensor(IMP[f"{c}__roles"]) - 1                  # reference 0 / 1 / 2 -> LOST / LONE / 1
    seed = int(IMP[f"{c}__shots_seed"][1])
    labels, fid = slot_outcomes(st, fates, U, torch.Generator().manual_seed(seed + 1))
    assert np.array_equal(labels.numpy(), IMP[f"{c}__labels"])
    assert np.array_equal(fid.numpy(), IMP[f"{c}__fid"])


def test_fixed_slot_state_keeps_one_operator_per_fixed_slot():
    from photonic_engines_b200.clifford.emitter import fixed_slot_state
    st, U, *_ = case("rand_n4_L2_t")
    fx = fixed_slot_state(st, [-1, 1, 2 + 3, -1], torch.as_tensor(U))
    assert np.allclose(fx.ops[0], st.ops[0]) and np.allclose(fx.ops[3], st.ops[3])
    assert np.allclose(fx.ops[1, 0], st.ops[1, 1]) and not fx.ops[1, 1].any()
    u = U[3, list(st.modes[2])]
    assert np.allclose(fx.ops[2, 0], np.einsum("l,lts->ts", u / np.linalg.norm(u), st.ops[2]))
    assert not fx.ops[2, 1].any()
