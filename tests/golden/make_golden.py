"""Generate the golden fixtures of the Fock sampling path from the REFERENCE implementation itself.

Run in a container where the reference project is importable (it is NOT needed at test time):

    python tests/golden/make_golden.py /path/to/photonic-engines [philox steps chains adaptive emitter slos emitter_imperfect]

It imports the reference read-only and records, with CPU tensors and the Triton CPU interpreter:

  philox.npz   tl.rand(seed, offset) bit patterns and the draw kernel's 48-bit uniforms, from a
               Triton kernel written here that calls tl.rand exactly as the reference's draw kernel
               does (photonic_engines/clifford/cofactors_triton.py:303-305).
  steps.npz    cofactors of blocks with repeated rows (variants.cofactors_2020, variants.py:96-114),
               the reference's extended-precision emulation of its kernel code
               (cuda_rect.rect_cofactors_emul, real="long double", form="fock", cuda_rect.py:959-985),
               and step amplitudes (variants.step_amplitudes, variants.py:176-194) on the
               reference's own test steps (tests/clifford/test_variants.py:41-49).
  adaptive.npz chains with a forced prefix and avoided modes: `_sample_streams(..., prefix=, avoid=)`
               rows and surviving stream ids with the sigma / seeds the generator produced, and
               `fock_sample(..., prefix=, avoid=, keep_ids=True)` occupations and ids (sampler.py:57-182,
               367-460).
  emitter.npz  EmitterMPS inputs (chi = 2): step weights of `emitter_reference.matrix_cofactor_weights`
               (emitter_reference.py:280-305) and occupations drawn by the exact torch sampler
               `emitter_sampler.sample_torch` (emitter_sampler.py:82-180) for seeded CPU generators.
  emitter_imperfect.npz  EmitterMPS occupations of the reference's emitter_sample with loss and partial
               distinguishability, and its slot outcomes (lost labels, lone rows, final spin).
  slos.npz     exact output probabilities of small circuits from the reference's SLOS kernel
               (slos/kernel.py:83-285): lossless, bunched input, x-model and lossy cases.
  chains.npz   whole chains drawn by the reference's sampler: `_sample_streams`
               (sampler.py:391-460) rows [S, n] in chain order, plus the sigma and per-step seeds
               the generator produced, and `fock_sample` occupations with loss / partial
               distinguishability (sampler.py:183-215) for a seeded CPU generator.
"""
from __future__ import annotations

import os
import sys

os.environ["TRITON_INTERPRET"] = "1"          # the reference's Triton kernels run on the CPU interpreter

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))


def haar(m: int, seed: int) -> torch.Tensor:
    """tests/helpers.py:10-17 of the reference (seeded QR of a complex Gaussian, phases fixed)."""
    g = torch.Generator().manual_seed(seed)
    z = torch.randn(m, m, generator=g, dtype=torch.float64) + 1j * torch.randn(m, m, generator=g, dtype=torch.float64)
    q, r = torch.linalg.qr(z)
    d = torch.diagonal(r)
    return q * (d / d.abs()).unsqueeze(0)


def make_philox():
    import triton
    import triton.language as tl

    @triton.jit
    def rand_kernel(out_ptr, seed, N: tl.constexpr):
        s = tl.arange(0, N)
        tl.store(out_ptr + s, tl.rand(seed, s))

    @triton.jit(do_not_specialize=["seed"])
    def uniform_kernel(out_ptr, seed):
        s = tl.program_id(0)
        two = tl.arange(0, 2)
        r = tl.rand(seed, s * 2 + two).to(tl.float64)
        u = tl.sum(tl.where(two == 0, r, r * 5.9604644775390625e-08), axis=0) / (1.0 + 5.9604644775390625e-08)
        tl.store(out_ptr + s, u)

    seeds = np.array([0, 1, 7, 12345, 2 ** 31 - 2, 987654321, 1804289383], dtype=np.int64)
    rand_bits = np.zeros((len(seeds), 128), dtype=np.uint32)
    unif = np.zeros((len(seeds), 96), dtype=np.float64)
    for i, sd in enumerate(seeds.tolist()):
        out = torch.zeros(128, dtype=torch.float32)
        rand_kernel[(1,)](out, sd, N=128)
        rand_bits[i] = out.numpy().view(np.uint32)
        u = torch.zeros(96, dtype=torch.float64)
        uniform_kernel[(96,)](u, sd)
        unif[i] = u.numpy()
    np.savez_compressed(os.path.join(HERE, "philox.npz"), seeds=seeds, rand_bits=rand_bits, uniforms=unif)


# the reference's own step cases (tests/clifford/test_variants.py:41-49) and collision patterns
# (tests/clifford/check_multi.py:22-30)
STEPS = [
    ([], [3]),
    ([4], [0, 0]),
    ([1, 1, 1], [2, 2, 0, 0]),
    ([0, 2, 2, 5], [0, 1, 1, 2, 3]),
    ([0, 1, 2, 3], [0, 1, 2, 3, 4]),
    ([2, 2, 2, 2], [0, 0, 0, 0, 1]),
    ([3, 3, 1, 0, 6, 6], [0, 1, 2, 3, 4, 5, 6]),
]
PATTERNS = [
    [0], [0, 0], [0, 1], [0, 0, 0], [1, 1, 0], [2, 1, 0], [0, 0, 0, 0], [1, 1, 0, 0], [3, 2, 1, 0], [2, 2, 1, 1],
    [0, 0, 0, 0, 0], [1, 1, 0, 0, 0], [2, 2, 1, 1, 0], [4, 3, 2, 1, 0], [1, 1, 1, 1, 0],
    [0] * 7, [1, 1, 1, 0, 0, 0, 2], [3, 3, 2, 2, 1, 1, 0], [6, 5, 4, 3, 2, 1, 0], [1, 1, 2, 2, 3, 3, 4],
    [0, 0, 1, 1, 2, 2, 3, 3, 4], [8, 7, 6, 5, 4, 3, 2, 1, 0], [1] * 9, [0, 0, 0, 0, 1, 1, 1, 2, 3],
    list(range(13)), [5, 5, 5, 3, 3, 1, 0, 0, 9, 9, 9, 9, 2],
]


def make_steps():
    from photonic_engines.clifford import cuda_rect
    from photonic_engines.clifford.variants import addends, cofactors_2020, step_amplitudes
    rng = np.random.default_rng(2024)
    blocks, rows_l, P64, Pld, T = [], [], [], [], []
    for rows in PATTERNS:
        K1 = len(rows)
        K = K1 + 1
        m = max(rows) + 1
        A = rng.normal(size=(m, K)) + 1j * rng.normal(size=(m, K))       # one row of A per output mode
        B = A[rows]                                                        # [K1, K]: equal modes -> equal rows
        P, t = cofactors_2020(torch.tensor(B), rows)
        Pl = cuda_rect.rect_cofactors_emul(torch.tensor(A[None]), torch.tensor([rows], dtype=torch.int64), K1,
                                           real="long double", form="fock")
        blocks.append(B); rows_l.append(rows); P64.append(P.numpy()); Pld.append(Pl[0].numpy()); T.append(t)
        assert t == addends("2020", rows, list(range(K)))
    # step amplitudes on the reference's test steps, U = haar(8, 1) (tests/clifford/test_variants.py:38-39)
    U8 = haar(8, 1)
    amps = [step_amplitudes(U8, r, c, "2020")[0].numpy() for r, c in STEPS]
    pad = max(len(b) for b in rows_l) + 1
    Bpad = np.zeros((len(blocks), pad - 1, pad), dtype=np.complex128)
    Rpad = np.full((len(blocks), pad - 1), -1, dtype=np.int64)
    P64p = np.zeros((len(blocks), pad), dtype=np.complex128)
    Pldp = np.zeros((len(blocks), pad), dtype=np.complex128)
    for i, (B, r, p, q) in enumerate(zip(blocks, rows_l, P64, Pld)):
        Bpad[i, : B.shape[0], : B.shape[1]] = B
        Rpad[i, : len(r)] = r
        P64p[i, : p.shape[0]] = p
        Pldp[i, : q.shape[0]] = q
    np.savez_compressed(
        os.path.join(HERE, "steps.npz"),
        blocks=Bpad, rows=Rpad, K1=np.array([len(r) for r in rows_l]), P_f64=P64p, P_ld=Pldp, addends=np.array(T),
        U8=U8.numpy(), step_rows=np.array([r + [-1] * (8 - len(r)) for r, _ in STEPS]),
        step_cols=np.array([c + [-1] * (8 - len(c)) for _, c in STEPS]),
        step_amps=np.array([np.pad(a, (0, 0)) for a in amps]))


# (name, m, in_modes, B circuits, shots, generator seed, U seed, algo)
CHAINS = [
    ("n4m8", 8, [0, 1, 2, 3], 1, 64, 3, 3, "auto"),
    ("bunched", 6, [0, 0, 2, 3], 1, 48, 11, 3, "2020"),
    ("n6m12", 12, [0, 1, 2, 3, 4, 5], 1, 48, 5, 1001, "auto"),
    ("batch2", 5, [0, 1, 2], 2, 24, 9, 21, "auto"),
    ("n7m10_2020", 10, [0, 1, 2, 3, 4, 5, 6], 1, 24, 17, 33, "2020"),
]
# public fock_sample with imperfections: (name, m, in_modes, shots, generator seed, U seed, loss, indist)
IMPERFECT = [
    ("loss05", 8, [0, 1, 2, 3, 4], 64, 1, 5, 0.5, None),
    ("indist095", 8, [0, 1, 2, 3, 4], 64, 2, 6, None, 0.95),
    ("loss07_indist08", 9, [0, 1, 2, 3, 4, 5], 48, 3, 7, 0.7, 0.8),
    ("indist_half_bunched", 7, [0, 0, 1, 2, 3], 48, 4, 8, None, 0.5),
]


def make_chains():
    from photonic_engines.clifford import fock_sample
    from photonic_engines.clifford import sampler as RS
    from photonic_engines.clifford.cofactors_triton import cofactor_partials_multi
    out = {}
    for name, m, in_modes, Bn, shots, gseed, useed, algo in CHAINS:
        U = torch.stack([haar(m, useed + b) for b in range(Bn)])
        n = len(in_modes)
        S = Bn * shots
        A2 = torch.view_as_real(U[:, :, in_modes].to(torch.complex128).contiguous())
        dp = torch.arange(Bn, dtype=torch.int64).repeat_interleave(shots)
        gen = torch.Generator().manual_seed(gseed)
        rows, _ = RS._sample_streams(A2, dp, n, m, gen, algo, 10, 1 << 16, 1 << 17, cofactor_partials_multi)
        g2 = torch.Generator().manual_seed(gseed)
        sig = torch.argsort(torch.rand(S, n, generator=g2), dim=1)
        seeds = torch.randint(0, 2 ** 31 - 1, (n,), generator=g2)
        occ = fock_sample(U if Bn > 1 else U[0], in_modes, shots, generator=torch.Generator().manual_seed(gseed),
                          algo=algo)
        out[f"{name}__U"] = U.numpy()
        out[f"{name}__in_modes"] = np.array(in_modes)
        out[f"{name}__meta"] = np.array([m, Bn, shots, gseed, useed])
        out[f"{name}__sigma"] = sig.numpy()
        out[f"{name}__seeds"] = seeds.numpy()
        out[f"{name}__rows"] = rows.numpy()
        out[f"{name}__occ"] = occ.numpy()
        print(name, "rows", rows.shape, flush=True)
    for name, m, in_modes, shots, gseed, useed, loss, indist in IMPERFECT:
        U = haar(m, useed)
        occ = fock_sample(U, in_modes, shots, generator=torch.Generator().manual_seed(gseed), loss=loss, indist=indist)
        out[f"{name}__U"] = U.numpy()
        out[f"{name}__in_modes"] = np.array(in_modes)
        out[f"{name}__meta"] = np.array([m, shots, gseed, useed])
        out[f"{name}__imperf"] = np.array([-1.0 if loss is None else loss, -1.0 if indist is None else indist])
        out[f"{name}__occ"] = occ.numpy()
        print(name, "occ", occ.shape, flush=True)
    np.savez_compressed(os.path.join(HERE, "chains.npz"), **out)


# (name, m, in_modes, B circuits, shots, generator seed, U seed, prefix, avoid, max_streams)
ADAPTIVE = [
    ("pre_shared", 8, [0, 1, 2, 3, 4, 5], 1, 40, 21, 51, [3, 3], None, 1 << 18),
    ("pre_avoid", 8, [0, 1, 2, 3, 4, 5], 1, 60, 22, 52, [2], [2, 5], 1 << 18),
    ("avoid_only", 7, [0, 1, 2, 3], 1, 60, 23, 53, None, [0, 4], 1 << 18),
    ("pre_batch", 6, [0, 1, 2, 3], 2, 30, 24, 54, [[1, 4], [2, 2]], [1, 2, 4], 1 << 18),
    ("pre_chunks", 7, [0, 1, 2, 3, 4], 1, 50, 25, 55, [6], [6, 0], 16),
    ("pre_full", 6, [0, 1, 2], 1, 12, 26, 56, [1, 1, 3], [0], 1 << 18),
]


def make_adaptive():
    from photonic_engines.clifford import fock_sample
    from photonic_engines.clifford import sampler as RS
    from photonic_engines.clifford.cofactors_triton import cofactor_partials_multi
    out = {}
    for name, m, in_modes, Bn, shots, gseed, useed, prefix, avoid, max_streams in ADAPTIVE:
        U = torch.stack([haar(m, useed + b) for b in range(Bn)])
        n = len(in_modes)
        S = Bn * shots
        A2 = torch.view_as_real(U[:, :, in_modes].to(torch.complex128).contiguous())
        dp = torch.arange(Bn, dtype=torch.int64).repeat_interleave(shots)
        pre_t = None if prefix is None else torch.as_tensor(prefix, dtype=torch.int64)
        mask = None
        if avoid is not None:
            mask = torch.zeros(m, dtype=torch.bool)
            mask[avoid] = True
        sig_l, seeds_l, rows_l, kept_l = [], [], [], []
        gen = torch.Generator().manual_seed(gseed)
        g2 = torch.Generator().manual_seed(gseed)
        for c0 in range(0, S, max_streams):
            dpc = dp[c0:c0 + max_streams].contiguous()
            rows, kept = RS._sample_streams(A2, dpc, n, m, gen, "auto", 10, 1 << 16, 1 << 17, cofactor_partials_multi,
                                            prefix=pre_t, avoid=mask)
            if pre_t is not None:
                sig = RS._prefix_order(A2, dpc, n, pre_t, g2)
            else:
                sig = torch.argsort(torch.rand(dpc.shape[0], n, generator=g2), dim=1)
            seeds_l.append(torch.randint(0, 2 ** 31 - 1, (n,), generator=g2))
            sig_l.append(sig)
            full = torch.full((dpc.shape[0], n), -1, dtype=torch.int64)
            ids = torch.arange(dpc.shape[0]) if kept is None else kept
            full[ids] = rows
            rows_l.append(full)
            alive = torch.zeros(dpc.shape[0], dtype=torch.bool)
            alive[ids] = True
            kept_l.append(alive)
        occ, oids = fock_sample(U if Bn > 1 else U[0], in_modes, shots, generator=torch.Generator().manual_seed(gseed),
                                prefix=prefix, avoid=avoid, keep_ids=True, max_streams=max_streams)
        out[f"{name}__U"] = U.numpy()
        out[f"{name}__in_modes"] = np.array(in_modes)
        out[f"{name}__meta"] = np.array([m, Bn, shots, gseed, useed, max_streams])
        out[f"{name}__prefix"] = np.array(prefix if prefix is not None else [], dtype=np.int64)
        out[f"{name}__avoid"] = np.array(avoid if avoid is not None else [], dtype=np.int64)
        out[f"{name}__sigma"] = torch.cat(sig_l).numpy()
        out[f"{name}__seeds"] = torch.stack(seeds_l).numpy()
        out[f"{name}__rows"] = torch.cat(rows_l).numpy()          # -1 rows: a stream dropped by `avoid`
        out[f"{name}__alive"] = torch.cat(kept_l).numpy()
        out[f"{name}__occ"] = occ.numpy()
        out[f"{name}__ids"] = oids.numpy()
        print(name, "occ", tuple(occ.shape), flush=True)
    np.savez_compressed(os.path.join(HERE, "adaptive.npz"), **out)


def _emitters():
    """(name, state) pairs: random emitters (chi = 2, 1 or 2 labels, projected or traced) and caterpillar
    states built by the reference's EmitterMPS.caterpillar (their arrays are what is stored)."""
    import math
    from photonic_engines import EmitterMPS, spin_gate
    out = []
    for name, n, L, seed, final in [("rand_n3_L2_f", 3, 2, 4, True), ("rand_n4_L2_t", 4, 2, 6, False),
                                    ("rand_n4_L1_f", 4, 1, 8, True), ("rand_n5_L2_f", 5, 2, 10, True),
                                    ("rand_n5_L1_t", 5, 1, 12, False)]:
        rng = np.random.default_rng(seed)
        ops = rng.normal(size=(n, L, 2, 2)) + 1j * rng.normal(size=(n, L, 2, 2))
        modes = tuple(tuple(range(k * L, (k + 1) * L)) for k in range(n))
        s0 = rng.normal(size=2) + 1j * rng.normal(size=2)
        f = (rng.normal(size=2) + 1j * rng.normal(size=2)) if final else None
        out.append((name, EmitterMPS(ops=ops, modes=modes, s0=s0, m=n * L + 1, final=f)))
    gates = [spin_gate(math.pi / 2, 0)] + [spin_gate(math.pi / 2, p) for p in (math.pi, 0, 0.9, 0.3)]
    out.append(("caterpillar_n5", EmitterMPS.caterpillar(5, gates)))
    out.append(("caterpillar_n4_f", EmitterMPS.caterpillar(4, gates[:4], final=(0.6, 0.8j))))
    return out


def make_emitter():
    from photonic_engines.clifford.emitter_reference import matrix_cofactor_weights
    from photonic_engines.clifford.emitter_sampler import sample_torch
    out = {}
    for si, (name, st) in enumerate(_emitters()):
        U = haar(st.m, 300 + si)
        out[f"{name}__ops"] = np.asarray(st.ops)
        out[f"{name}__modes"] = np.array([list(mk) for mk in st.modes])
        out[f"{name}__s0"] = np.asarray(st.s0)
        out[f"{name}__final"] = np.asarray(st.final) if st.final is not None else np.zeros(0, dtype=np.complex128)
        out[f"{name}__m"] = np.array([st.m])
        out[f"{name}__U"] = U.numpy()
        rng = np.random.default_rng(50 + si)
        Ts, rows_l, fins, ws = [], [], [], []
        for _ in range(4):                                   # steps with k = 1 .. n placed photons
            k = int(rng.integers(1, st.n + 1))
            T = sorted(rng.choice(st.n, size=k, replace=False).tolist())
            rows = rng.integers(0, st.m, size=k - 1).tolist()
            fin = None if st.final is not None else torch.eye(2, dtype=torch.complex128)[int(rng.integers(0, 2))]
            w, _ = matrix_cofactor_weights(U, st, T, rows, final=fin)
            Ts.append(T + [-1] * (st.n - k)); rows_l.append(rows + [-1] * (st.n - k))
            fins.append(-1 if fin is None else int(torch.argmax(fin.abs())))
            ws.append(w.numpy())
        out[f"{name}__step_T"] = np.array(Ts); out[f"{name}__step_rows"] = np.array(rows_l)
        out[f"{name}__step_final"] = np.array(fins); out[f"{name}__step_w"] = np.array(ws)
        shots, seed = 300, 7 + si
        occ = sample_torch(st, U, shots, generator=torch.Generator().manual_seed(seed))
        out[f"{name}__shots_seed"] = np.array([shots, seed])
        out[f"{name}__occ"] = occ.numpy()
        print(name, "emitter", tuple(occ.shape), flush=True)
    np.savez_compressed(os.path.join(HERE, "emitter.npz"), **out)


# (emitter, loss eta or None, x-model overlap or None, unravel): imperfect emitter draws recorded
EMITTER_IMPERFECT = [("rand_n4_L2_t", 0.7, None, True), ("rand_n4_L2_t", None, 0.8, True),
                     ("rand_n5_L2_f", 0.8, 0.9, True), ("caterpillar_n5", 0.75, None, True),
                     ("caterpillar_n5", 0.7, None, False), ("rand_n5_L1_t", 0.85, 0.85, True)]


def make_emitter_imperfect():
    """emitter_imperfect.npz: occupations of the reference's emitter_sample with loss and / or x-model
    partial distinguishability (photonic_engines/clifford/__init__.py:36-128, backend "torch", seeded CPU
    generators), and the slot outcomes of emitter_terms.sample_slot_outcomes (emitter_terms.py:71-137) for
    recorded fates (0 lost, 1 lone, 2 interfering)."""
    from photonic_engines.clifford import emitter_sample
    from photonic_engines.clifford.emitter_terms import sample_slot_outcomes
    states = dict(_emitters())
    out = {}
    for ci, (name, eta, x, unravel) in enumerate(EMITTER_IMPERFECT):
        st = states[name]
        U = haar(st.m, 700 + ci)
        case = f"c{ci}"
        out[f"{case}__name"] = np.array(name)
        out[f"{case}__U"] = U.numpy()
        out[f"{case}__imperf"] = np.array([-1.0 if eta is None else eta, -1.0 if x is None else x, float(unravel)])
        shots, seed = 200, 40 + ci
        occ = emitter_sample(st, U, shots, generator=torch.Generator().manual_seed(seed), backend="torch",
                             loss=eta, indist=x, unravel=unravel)
        out[f"{case}__shots_seed"] = np.array([shots, seed])
        out[f"{case}__occ"] = occ.numpy()
        rng = np.random.default_rng(90 + ci)
        roles = torch.as_tensor(rng.choice([0, 1, 2], size=(64, st.n), p=[0.3, 0.2, 0.5]), dtype=torch.long)
        labels, fid = sample_slot_outcomes(st, roles, U, generator=torch.Generator().manual_seed(seed + 1))
        out[f"{case}__roles"] = roles.numpy()
        out[f"{case}__labels"] = labels.numpy()
        out[f"{case}__fid"] = fid.numpy()
        print(case, name, eta, x, unravel, tuple(occ.shape), int(occ.sum()), flush=True)
    np.savez_compressed(os.path.join(HERE, "emitter_imperfect.npz"), **out)


# (name, m, input modes, Haar seed, loss eta or None, x-model overlap or None): the small cases whose exact
# law the tests compare samples with (histogram TVD tests), lossless, lossy and partially distinguishable
SLOS_CASES = [("m4_n3", 4, [0, 1, 2], 104, None, None), ("m5_bunched", 5, [0, 0, 1], 105, None, None),
              ("m6_n4", 6, [0, 1, 2, 3], 106, None, None), ("m5_n3_x07", 5, [0, 1, 2], 55, None, 0.7),
              ("m4_n3_loss06", 4, [0, 1, 2], 5, 0.6, None)]


def make_slos():
    """slos.npz: exact output probabilities from the reference's SLOS kernel (FockSLOSKernel.probs,
    photonic_engines/slos/kernel.py:83-285, complex128; `indist=` its x-mixture, `loss=` its thinned
    LossyDistribution) on Haar circuits built as the oracle builds them (the oracle's haar_unitary, which
    restates tests/helpers.py:10-17)."""
    from photonic_engines.slos.kernel import FockSLOSKernel
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.oracle import haar_unitary
    out = {}
    for name, m, modes, seed, eta, x in SLOS_CASES:
        U = torch.as_tensor(haar_unitary(m, seed))
        occ_in = [modes.count(j) for j in range(m)]
        ker = FockSLOSKernel(len(modes), m, occ_in, dtype=torch.complex128)
        if eta is not None:
            d = ker.probs(U, loss=eta).as_dict()
            states = np.array([list(k) for k in d], dtype=np.int64)
            probs = np.array([float(v) for v in d.values()])
        else:
            probs = ker.probs(U, indist=x).numpy() if x is not None else ker.probs(U).numpy()
            states = np.array(ker.layers.final_states, dtype=np.int64)
        out[f"{name}__meta"] = np.array([m, seed, -1.0 if eta is None else eta, -1.0 if x is None else x])
        out[f"{name}__modes"] = np.array(modes, dtype=np.int64)
        out[f"{name}__states"] = states
        out[f"{name}__probs"] = probs
        print(name, "slos", states.shape, float(probs.sum()), flush=True)
    np.savez_compressed(os.path.join(HERE, "slos.npz"), **out)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PE_REFERENCE", "")
    if not ref or not os.path.isdir(ref):
        raise SystemExit("usage: make_golden.py /path/to/photonic-engines (the reference checkout)")
    sys.path.insert(0, ref)
    parts = sys.argv[2:] or ["philox", "steps", "chains", "adaptive"]
    for part in parts:
        {"philox": make_philox, "steps": make_steps, "chains": make_chains, "adaptive": make_adaptive,
         "emitter": make_emitter, "slos": make_slos, "emitter_imperfect": make_emitter_imperfect}[part]()
        print(part, "done", flush=True)
