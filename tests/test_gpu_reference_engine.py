"""Sample-for-sample parity with the reference's own GPU engine on the same GPU.

The reference's offline install (baseline/_ref, its public `photonic_engines.clifford.fock_sample` with its
default Triton backend, unmodified) and this library's `fock_sample` are called with equal CUDA generators
at the benchmark shapes: the occupations must be identical row for row — the same sigma draws, the same
loss / distinguishability partition, the same Philox uniforms and the same picks.  Skipped when the
reference is not installed beside the repository or its Triton kernels cannot be built.
(The reference's own cross-path checks work the same way: tests/clifford/check_algos_gpu.py:54-72,
check_single.py:19-33.)"""
import os
import sys

import numpy as np
import pytest
import torch

from oracle import oracle as O
from photonic_engines_b200.clifford import fock_sample

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "baseline", "_ref")
DEV = "cuda"


@pytest.fixture(scope="module")
def ref():
    if not os.path.isdir(os.path.join(REF, "photonic_engines")):
        pytest.skip("the reference is not installed in baseline/_ref")
    pytest.importorskip("triton")
    sys.path.insert(0, REF)
    try:
        import photonic_engines.clifford as rc
    finally:
        sys.path.remove(REF)
    return rc.fock_sample


def _gen(seed):
    return torch.Generator(device=DEV).manual_seed(seed)


def _same(ref_fn, U, modes, shots, seed, **kw):
    a = ref_fn(U, modes, shots, generator=_gen(seed), **kw)
    b = fock_sample(U, modes, shots, generator=_gen(seed), **kw)
    assert a.shape == b.shape
    diff = int((a.cpu() != b.cpu()).any(dim=1).sum())
    assert diff == 0, f"{diff} of {a.shape[0]} rows differ"
    return b


@pytest.mark.parametrize("precision", ["f64", "mixed", "compensated"])
def test_n20_m400_lossless(ref, precision):
    U = torch.tensor(O.haar_unitary(400, 1002), device=DEV)
    a = ref(U, list(range(20)), 300, generator=_gen(11))
    b = fock_sample(U, list(range(20)), 300, generator=_gen(11), precision=precision)
    assert torch.equal(a, b)


def test_n30_m900_loss_half(ref):
    """Ragged survivors k ~ Bin(30, 0.5) in length tiers."""
    U = torch.tensor(O.haar_unitary(900, 3001), device=DEV)
    occ = _same(ref, U, list(range(30)), 3000, 12, loss=0.5)
    assert (occ.sum(1) <= 30).all()


def test_n28_m784_partial_distinguishability(ref):
    U = torch.tensor(O.haar_unitary(784, 4001), device=DEV)
    occ = _same(ref, U, list(range(28)), 12, 13, indist=0.95)
    assert (occ.sum(1) == 28).all()


def test_small_circuits_with_loss(ref):
    """Every 32nd of the 256 small circuits of the many-instance configuration, each with its own eta."""
    rng = np.random.default_rng(5000)
    for i in range(256):
        m = int(rng.choice([16, 24, 32, 48, 64]))
        n = int(rng.integers(4, min(12, m // 4) + 1))
        eta = float(rng.uniform(0.6, 1.0))
        if i % 32 == 0:
            U = torch.tensor(O.haar_unitary(m, 5000 + i), device=DEV)
            _same(ref, U, list(range(n)), 1000, 100 + i, loss=eta)


def test_repeated_input_modes_with_loss_and_distinguishability(ref):
    U = torch.tensor(O.haar_unitary(24, 77), device=DEV)
    modes = [0, 0, 1, 3, 3, 3, 5, 8]
    _same(ref, U, modes, 500, 14)
    _same(ref, U, modes, 500, 15, loss=0.7)
    _same(ref, U, modes, 500, 16, loss=0.8, indist=0.9)


def test_batched_circuits_with_per_circuit_shots(ref):
    U = torch.stack([torch.tensor(O.haar_unitary(32, 200 + b), device=DEV) for b in range(3)])
    _same(ref, U, list(range(10)), 64, 17)
    _same(ref, U, list(range(10)), torch.tensor([5, 0, 40]), 18)


def test_prefix_and_avoid(ref):
    U = torch.tensor(O.haar_unitary(40, 78), device=DEV)
    a, ia = ref(U, list(range(10)), 400, generator=_gen(19), prefix=[0, 1], avoid=[2, 3], keep_ids=True)
    b, ib = fock_sample(U, list(range(10)), 400, generator=_gen(19), prefix=[0, 1], avoid=[2, 3], keep_ids=True)
    assert torch.equal(ia.cpu(), ib.cpu()) and torch.equal(a.cpu(), b.cpu())


def test_single_sample_and_short_chains(ref):
    """One shot per call (the split latency path) and the n = 6, m = 12 workload (warp form)."""
    U = torch.tensor(O.haar_unitary(400, 1002), device=DEV)
    for seed in (21, 22, 23):
        _same(ref, U, list(range(20)), 1, seed)
    U12 = torch.tensor(O.haar_unitary(12, 1001), device=DEV)
    _same(ref, U12, list(range(6)), 10000, 24)


@pytest.fixture(scope="module")
def ref_emitter():
    if not os.path.isdir(os.path.join(REF, "photonic_engines")):
        pytest.skip("the reference is not installed in baseline/_ref")
    pytest.importorskip("triton")
    sys.path.insert(0, REF)
    try:
        import photonic_engines.clifford as rc
        from photonic_engines.states import EmitterMPS, spin_gate
    finally:
        sys.path.remove(REF)
    return rc.emitter_sample, EmitterMPS, spin_gate


@pytest.mark.parametrize("kw", [{}, {"loss": 0.8}, {"loss": 0.8, "unravel": False}, {"indist": 0.9}])
def test_emitter_caterpillar(ref_emitter, kw):
    """The linear cluster state of 8 photons in 16 modes, emitter traced, through both emitter_sample calls
    with equal CPU generator seeds (the generator the reference's emitter path draws its host choices from)."""
    import math

    from photonic_engines_b200.clifford import emitter_sample
    from photonic_engines_b200.states import caterpillar, spin_gate
    ref_fn, EmitterMPS, ref_gate = ref_emitter
    n, m = 8, 16
    U = torch.tensor(O.haar_unitary(m, 88), device=DEV)
    rst = EmitterMPS.caterpillar(n, [ref_gate(math.pi / 2, 0)] * n, m=m)
    st = caterpillar(n, [spin_gate(math.pi / 2, 0)] * n, m=m)
    a = ref_fn(rst, U, 256, generator=torch.Generator().manual_seed(31), **kw)
    b = emitter_sample(st, U, 256, generator=torch.Generator().manual_seed(31), **kw)
    assert torch.equal(a.cpu(), b.cpu())


def test_lossy_call_with_long_survivors_runs_the_split_tier(ref):
    """n_in = 30, m = 900 at transmission 0.9: most survivors have more than 24 photons, so the call's longest
    tier runs with split steps (kernels.tier_plan mode 2) beside the 21-24- and 17-20-photon tiers."""
    from photonic_engines_b200.clifford import kernels as K
    U = torch.tensor(O.haar_unitary(900, 3002), device=DEV)
    tiers = K.tier_plan({27: 20, 26: 10, 23: 5, 19: 2}, 30, "f64", torch.device(DEV))
    assert tiers[0][3] == 2
    _same(ref, U, list(range(30)), 48, 25, loss=0.9)
