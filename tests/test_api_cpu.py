"""`fock_sample` argument checks and the absence of any CPU path (the reference's error behaviour:
photonic_engines/clifford/sampler.py:96-135, tests/clifford/test_fock_sampler_cpu.py:113-121)."""
import pytest
import torch

from oracle import oracle as O
from photonic_engines_b200 import FockState
from photonic_engines_b200 import _native as N
from photonic_engines_b200.clifford import fock_sample, sample
from photonic_engines_b200.imperfections import Distinguishability, as_model

U4 = torch.as_tensor(O.haar_unitary(4, 13))


@pytest.mark.parametrize(("kw", "match"), [({"backend": "nope"}, "unknown backend"),
                                           ({"backend": "torch"}, "unknown backend"),
                                           ({"algo": "2019"}, "unknown algo"),
                                           ({"precision": "f16"}, "unknown precision")])
def test_an_unknown_backend_algo_or_precision_is_rejected(kw, match):
    with pytest.raises(ValueError, match=match):
        fock_sample(U4, [0, 1], 8, generator=torch.Generator().manual_seed(0), **kw)


def test_input_algo_with_the_cuda_backend_is_not_implemented():
    with pytest.raises(NotImplementedError):
        fock_sample(U4, [0, 1], 2, backend="cuda", algo="input")


def test_exq_backend_is_not_part_of_the_library():
    with pytest.raises(NotImplementedError):
        fock_sample(U4, [0, 1], 2, backend="exq")


def test_there_is_no_cpu_path():
    """A CPU tensor is refused instead of being sampled by anything but the CUDA kernels."""
    with pytest.raises((N.NativeError, ValueError)):
        fock_sample(U4, [0, 1], 2, generator=torch.Generator().manual_seed(0))


def test_sample_refuses_other_input_types():
    with pytest.raises(TypeError):
        sample(object(), U4, 2)
    assert FockState((1, 0, 2)).modes() == [0, 2, 2]


def test_indist_model_normalisation():
    assert as_model(None) is None and as_model(1.0) is None
    assert as_model(0.9) == Distinguishability(x=0.9)
    assert as_model([1.0, 0.8, 0.95]) == Distinguishability(x=0.8)
    assert as_model(Distinguishability(species=(1.0,))) is None
    assert Distinguishability.from_hom_visibility(0.81) == Distinguishability(x=0.9)
    with pytest.raises(ValueError):
        as_model(1.5)
    with pytest.raises(ValueError):
        Distinguishability(x=0.5, species=(0.2,))
    with pytest.raises(ValueError):
        Distinguishability(species=(0.7, 0.4))


def test_photon_limits_are_checked_on_the_host():
    """64 photons in FP64, 32 in the mixed form (its FP32 error grows ~1.35x per column); the C ABI
    answers PE_ERR_SIZE beyond them, the host refuses first with a clear message."""
    N.check_photons(64, "f64")
    N.check_photons(32, "mixed")
    with pytest.raises(ValueError, match="at most 64"):
        N.check_photons(65, "f64")
    with pytest.raises(ValueError, match="mixed"):
        N.check_photons(33, "mixed")
    from photonic_engines_b200.clifford.kernels import default_tpl
    assert [default_tpl(n, "f64") for n in (6, 18, 24, 32, 36, 48, 64)] == [1, 1, 2, 2, 2, 4, 4]
    assert [default_tpl(n, "mixed") for n in (6, 18, 24, 32)] == [1, 1, 2, 2]
    assert [default_tpl(n, "compensated") for n in (6, 18, 24, 32)] == [1, 2, 4, 4]
    N.check_photons(32, "compensated")
    with pytest.raises(ValueError, match="compensated"):
        N.check_photons(33, "compensated")
