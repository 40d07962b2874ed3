"""The reference's own callers of the sampling path, driven by this library.

`AdaptiveCircuit.sample` (photonic_engines/adaptive.py:582-640: forced-prefix and rejection final stages,
with loss) and `NonlinearCircuit.sample` (photonic_engines/nonlinear.py:471-530: branch proposals of U_b
batches with per-circuit shots) take a `base_sampler` hook in place of their stock `fock_sample` call.
Run from the reference's unmodified offline install (baseline/_ref) once with the stock Triton backend and
once with this library's `fock_sample` behind the hook, from equal CUDA generator seeds, they must return
the same samples.  Skipped when the reference is not installed beside the repository."""
import os
import sys

import pytest
import torch

from oracle import oracle as O
from photonic_engines_b200.clifford import fock_sample

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "baseline", "_ref")
DEV = "cuda"


@pytest.fixture(scope="module")
def refmods():
    if not os.path.isdir(os.path.join(REF, "photonic_engines")):
        pytest.skip("the reference is not installed in baseline/_ref")
    pytest.importorskip("triton")
    sys.path.insert(0, REF)
    try:
        from photonic_engines.adaptive import AdaptiveCircuit
        from photonic_engines.nonlinear import NonlinearCircuit
    finally:
        sys.path.remove(REF)
    return AdaptiveCircuit, NonlinearCircuit


def _haar(m, seed):
    return torch.tensor(O.haar_unitary(m, seed), device=DEV)


def _gen(seed):
    return torch.Generator(device=DEV).manual_seed(seed)


M, T_IN, LEVELS = 10, [0, 2, 4, 6], [[1], [3, 5]]


def _policy(lam, p):
    """A Haar unitary on the unmeasured modes, different for every outcome prefix (deterministic)."""
    size = M - (1 if lam == 1 else 3)
    return _haar(size, 300 + 13 * lam + sum(int(x) * 7 ** i for i, x in enumerate(p)))


def _prefix_base(U, in_modes, shots, generator, prefix, avoid):
    return fock_sample(U, in_modes, shots, generator=generator, prefix=prefix, avoid=avoid,
                       keep_ids=isinstance(shots, torch.Tensor))


def _plain_base(U, in_modes, shots, generator):
    return fock_sample(U, in_modes, shots, generator=generator)


@pytest.mark.parametrize(("final", "chain", "loss"), [("prefix", "marginal", None), ("prefix", "rejection", None),
                                                      ("prefix", "marginal", 0.8), ("clifford", "marginal", None)])
def test_adaptive_circuit(refmods, final, chain, loss):
    AdaptiveCircuit = refmods[0]
    U0 = _haar(M, 31)
    base = _prefix_base if final == "prefix" else _plain_base
    a = AdaptiveCircuit(U0, T_IN, LEVELS, _policy).sample(600, generator=_gen(41), chain=chain, final=final, loss=loss)
    b = AdaptiveCircuit(U0, T_IN, LEVELS, _policy).sample(600, generator=_gen(41), chain=chain, final=final, loss=loss,
                                                          base_sampler=base)
    assert a.shape == b.shape and torch.equal(a.cpu(), b.cpu())


@pytest.mark.parametrize("loss", [None, 0.85])
def test_nonlinear_circuit(refmods, loss):
    NonlinearCircuit = refmods[1]
    Us = [_haar(12, 50 + i) for i in range(3)]
    sites = [(1, 2, 0.7), (1, 5, 0.3), (2, 1, [0.2, 1.3, -0.4, 0.9, 0.0, 2.2])]
    a = NonlinearCircuit(Us, [0, 1, 3, 4, 7], sites).sample(500, generator=_gen(43), loss=loss)
    b = NonlinearCircuit(Us, [0, 1, 3, 4, 7], sites).sample(500, generator=_gen(43), loss=loss,
                                                            base_sampler=lambda U, t, s, g: fock_sample(U, t, s, generator=g))
    assert a.shape == b.shape and torch.equal(a.cpu(), b.cpu())
