"""B200-native (sm_100a) exact Fock boson sampler: the Clifford & Clifford sampling path of
photonic-engines behind its `clifford.fock_sample` API, computed by hand-written CUDA kernels
(libpe_b200.so, C ABI in include/pe_b200.h)."""
from . import clifford, imperfections, states
from .states import EmitterMPS, FockState

__version__ = "0.1.0"
__all__ = ["EmitterMPS", "FockState", "clifford", "imperfections", "states"]
