"""Build of the CUDA library `libpe_b200.so` (in-tree, next to this file) for sm_100a.

Every kernel variant (precision x threads per Gray lane x largest column tier) is one object file
compiled from csrc/fock_inst.cu with its own -D flags, in parallel; csrc/fock_api.cu holds the C ABI.
Objects are rebuilt only when a source is newer.  `python -m photonic_engines_b200.build` builds it.
Environment: PE_NVCC_FLAGS (extra nvcc flags, e.g. tuning macros), PE_BUILD_DIR (object directory),
PE_LIB (output library path; the loader reads the same variable).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.environ.get("PE_BUILD_DIR", os.path.join(HERE, "_build"))
LIB = os.environ.get("PE_LIB", os.path.join(HERE, "libpe_b200.so"))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
         *os.environ.get("PE_NVCC_FLAGS", "").split()]

# (precision 0 FP64 / 1 mixed / 2 compensated, threads per lane, largest tier) of every compiled chain/cofactor kernel pair
VARIANTS = [(mx, tpl, kpm) for mx in (0, 1) for tpl, kpms in ((1, (8, 16, 20)), (2, (8, 16, 20, 24, 28, 32)),
                                                              (4, (8, 16, 20, 24, 28, 32))) for kpm in kpms]
VARIANTS += [(0, 2, 40)] + [(0, 4, kpm) for kpm in (40, 48, 56, 64)]      # beyond 32 photons: FP64 only
# compensated mixed form (double-float state: 12 FP32 pairs per column pair): two-thread lanes up to 20
# columns, four-thread lanes beyond
VARIANTS += [(2, 1, 8)] + [(2, 2, kpm) for kpm in (8, 16, 20)] + [(2, 4, kpm) for kpm in (24, 28, 32)]
if os.environ.get("PE_VARIANTS"):          # a subset "m,t,k;m,t,k" (experiments: smaller, faster builds)
    VARIANTS = [tuple(int(x) for x in v.split(",")) for v in os.environ["PE_VARIANTS"].split(";")]


def variant_flags(mx: int, tpl: int, kpm: int) -> list[str]:
    """Lanes that hold many columns per thread (one-thread lanes of 16 and 20 columns, two-thread lanes of
    24 to 40, four-thread lanes of 40 to 64) are compiled for 128-thread CTAs, two per SM, so that every
    thread may use 255 registers;
    the others for 256-thread CTAs at 128 registers.  Two-thread lanes at 24-32 columns compiled this way
    run 1.1-1.9x faster than four-thread lanes at 128 registers (FP64, m = 2n).  The compensated form keeps
    a double-float column sum, accumulator and prefix product per column: its two-thread lanes from 16
    columns and four-thread lanes from 24 get the 255-register allocation too."""
    if (tpl == 1 and kpm >= 16) or (tpl == 2 and kpm >= 24) or (tpl == 4 and kpm > 32):
        return ["-DPE_MAXT=128", "-DPE_MINB=2"]
    if mx == 2 and ((tpl == 2 and kpm >= 16) or (tpl == 4 and kpm >= 24)):
        return ["-DPE_MAXT=128", "-DPE_MINB=2"]
    return []


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h"))] + \
        [os.path.join(ROOT, "include", "pe_b200.h"), os.path.abspath(__file__)]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build(jobs: int | None = None, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every variant and link the library; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    deps = _sources()
    tasks = []
    for mx, tpl, kpm in VARIANTS:
        obj = os.path.join(OBJ, f"fock_m{mx}_t{tpl}_k{kpm}.o")
        if _stale(obj, deps):
            tasks.append([NVCC, *ARCH, *FLAGS, *(["-Xptxas", "-v"] if ptxas_info else []), f"-DPE_MIXED={mx}",
                          f"-DPE_TPL={tpl}", f"-DPE_KPM={kpm}", *variant_flags(mx, tpl, kpm), "-c",
                          os.path.join(CSRC, "fock_inst.cu"), "-o", obj])
    extra = []
    for name in ("fock_api", "fock_batch", "emitter"):
        obj = os.path.join(OBJ, f"{name}.o")
        extra.append(obj)
        if _stale(obj, deps):
            tasks.append([NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, f"{name}.cu"), "-o", obj])
    objs = [os.path.join(OBJ, f"fock_m{mx}_t{tpl}_k{kpm}.o") for mx, tpl, kpm in VARIANTS] + extra
    if tasks:
        with ThreadPoolExecutor(jobs or os.cpu_count() or 4) as ex:
            for out in ex.map(_run, tasks):
                if verbose and out.strip():
                    print(out)
    if tasks or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
