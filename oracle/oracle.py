"""CPU oracle of the Clifford & Clifford Fock sampler: ctypes binding of `liboracle.so` plus the
small exact references (Ryser permanents, exact output distributions, Haar unitaries).

TEST INFRASTRUCTURE.  Only `tests/`, `__graft_entry__.smoke()` and `bench.py`'s CPU-baseline arm
may import this module; the product path (`photonic_engines_b200`) never does.

What it restates (file:line in the reference project):
  chain over steps, stream layout        photonic_engines/clifford/sampler.py:391-460
  multiplicity tables / halving          photonic_engines/clifford/cofactors_triton.py:413-447
  Gray odometer                          photonic_engines/clifford/cuda_cofactors.py:72-106
  2020 cofactors, exact all-but-one      photonic_engines/clifford/variants.py:70-114
  amplitudes, 48-bit uniform, pick rule  photonic_engines/clifford/cofactors_triton.py:287-308
  Philox4x32-10 as tl.rand calls it      triton/language/random.py (installed Triton)
  forced prefix / avoided modes          photonic_engines/clifford/sampler.py:391-460 (adaptive_chains)
  Ryser permanent                        tests/clifford/check_cofactors.py:17-24
  exact output distribution              tests/clifford/check_sampler.py:25-37
  Haar unitary                           tests/helpers.py:10-17
"""
from __future__ import annotations

import ctypes
import itertools
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file (gcc).  Returns its path."""
    src = [os.path.join(_HERE, f) for f in ("fock_oracle.c", "oracle_impl.h", "Makefile")]
    if force or not os.path.exists(_LIB_PATH) or any(os.path.getmtime(f) > os.path.getmtime(_LIB_PATH) for f in src):
        env = dict(os.environ)
        env["CC"] = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else env.get("CC", "gcc")
        subprocess.run(["make", "-s", "-B", "-C", _HERE], check=True, env=env)
    return _LIB_PATH


def lib():
    """The loaded oracle library (built on first use when missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_philox_randint.restype = ctypes.c_uint32
        L.oracle_philox_randint.argtypes = [ctypes.c_uint64, ctypes.c_uint32]
        L.oracle_triton_rand.restype = ctypes.c_float
        L.oracle_triton_rand.argtypes = [ctypes.c_uint64, ctypes.c_uint32]
        L.oracle_uniform.restype = ctypes.c_double
        L.oracle_uniform.argtypes = [ctypes.c_uint64, ctypes.c_int64]
        L.oracle_uniforms.restype = None
        L.oracle_uniforms.argtypes = [_i64p, ctypes.c_int, ctypes.c_int64, _f64p]
        for nm in ("oracle_cofactors_f64", "oracle_cofactors_ld"):
            f = getattr(L, nm)
            f.restype = ctypes.c_int64
            f.argtypes = [_f64p, _i64p, ctypes.c_int, ctypes.c_int, _f64p]
        L.oracle_addends.restype = ctypes.c_int64
        L.oracle_addends.argtypes = [_i64p, ctypes.c_int]
        for nm in ("oracle_step_f64", "oracle_step_ld"):
            f = getattr(L, nm)
            f.restype = ctypes.c_int64
            f.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, _i64p, _i64p, ctypes.c_int, ctypes.c_double, _f64p, _f64p]
        for nm in ("oracle_chain_f64", "oracle_chain_ld"):
            f = getattr(L, nm)
            f.restype = ctypes.c_int
            f.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64p, _i64p, _f64p,
                          ctypes.c_int64, _i64p, _f64p, _f64p, _i64p, ctypes.c_int]
        _lib = L
    return _lib


def _p64(a):
    return a.ctypes.data_as(_f64p)


def _pi64(a):
    return a.ctypes.data_as(_i64p)


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128))


# ---------------------------------------------------------------------------------------- RNG

def philox_randint(seed: int, offset: int) -> int:
    """randint4x(seed, offset)[0] of Triton's Philox4x32-10 (uint32)."""
    return int(lib().oracle_philox_randint(seed, offset))


def triton_rand(seed: int, offset: int) -> float:
    """tl.rand(seed, offset) for an int32 offset: float32 in [0, 1)."""
    return float(lib().oracle_triton_rand(seed, offset))


def uniforms(seeds, S: int) -> np.ndarray:
    """u [S, n]: the draw kernel's 48-bit uniform of stream s at step k (seed seeds[k])."""
    seeds = np.ascontiguousarray(np.asarray(seeds, dtype=np.int64))
    out = np.empty((S, seeds.shape[0]), dtype=np.float64)
    lib().oracle_uniforms(_pi64(seeds), seeds.shape[0], S, _p64(out))
    return out


# ---------------------------------------------------------------------------------------- steps

def cofactors(B, rows, precision: str = "f64") -> tuple[np.ndarray, int]:
    """P [K] = per(B without column c) for B [K1, K] complex (rows: chosen modes, repeats allowed)."""
    B = _c128(B)
    K1, K = B.shape
    rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int64).reshape(-1))
    P = np.empty(K, dtype=np.complex128)
    f = lib().oracle_cofactors_f64 if precision == "f64" else lib().oracle_cofactors_ld
    T = f(_p64(B.view(np.float64)), _pi64(rows), K1, K, _p64(P.view(np.float64)))
    if T < 0:
        raise ValueError("oracle cofactors: bad sizes")
    return P, int(T)


def addends(rows) -> int:
    """Addend count of a step whose chosen rows are `rows` (2020 closed form)."""
    rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int64).reshape(-1))
    return int(lib().oracle_addends(_pi64(rows), rows.shape[0]))


def step(A, rows, cols, u: float, precision: str = "f64") -> tuple[int, np.ndarray, float]:
    """One chain step: (pick, weights w [m], gap).  A [m, n] complex, rows the k-1 chosen modes,
    cols the k input columns sigma(1..k) (indices into A's columns)."""
    A = _c128(A)
    m, n = A.shape
    rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int64).reshape(-1))
    cols = np.ascontiguousarray(np.asarray(cols, dtype=np.int64).reshape(-1))
    k = cols.shape[0]
    full_rows = np.zeros(max(k, 1), dtype=np.int64)
    full_rows[: rows.shape[0]] = rows
    w = np.empty(m, dtype=np.float64)
    gap = ctypes.c_double(0.0)
    f = lib().oracle_step_f64 if precision == "f64" else lib().oracle_step_ld
    idx = f(_p64(A.view(np.float64)), m, n, _pi64(full_rows), _pi64(cols), k, float(u), _p64(w), ctypes.byref(gap))
    if idx < 0:
        raise ValueError("oracle step: bad sizes")
    return int(idx), w, float(gap.value)


def chain(A, dp, sigma, u, precision: str = "f64", marg: bool = False, threads: int = 0):
    """Whole chains: A [G, m, n] complex (input columns per instance), dp [S], sigma [S, k] (column indices
    < n, k <= n steps), u [S, k].  Returns dict(rows [S, k], gap [S, k], addends [S], marg [S, k, m] or None)."""
    A = _c128(A)
    if A.ndim == 2:
        A = A[None]
    G, m, n = A.shape
    dp = np.ascontiguousarray(np.asarray(dp, dtype=np.int64).reshape(-1))
    S = dp.shape[0]
    sigma = np.ascontiguousarray(np.asarray(sigma, dtype=np.int64).reshape(S, -1))
    k = sigma.shape[1]
    u = np.ascontiguousarray(np.asarray(u, dtype=np.float64).reshape(S, k))
    rows = np.zeros((S, k), dtype=np.int64)
    gap = np.zeros((S, k), dtype=np.float64)
    add = np.zeros(S, dtype=np.int64)
    mg = np.zeros((S, k, m), dtype=np.float64) if marg else None
    if S == 0:
        return {"rows": rows, "gap": gap, "addends": add, "marg": mg}
    f = lib().oracle_chain_f64 if precision == "f64" else lib().oracle_chain_ld
    rc = f(_p64(A.view(np.float64)), G, m, n, k, _pi64(dp), _pi64(sigma), _p64(u), S, _pi64(rows),
           _p64(mg) if marg else None, _p64(gap), _pi64(add), int(threads))
    if rc != 0:
        raise ValueError("oracle chain: bad sizes or instance ids")
    return {"rows": rows, "gap": gap, "addends": add, "marg": mg}


def adaptive_chains(A, dp, sigma, prefix_rows, seeds, seed_row, rng_off0, avoid=None,
                    precision: str = "f64") -> tuple[np.ndarray, np.ndarray]:
    """Chains with a forced prefix and avoided modes, stream by stream in the reference's step order
    (sampler.py:391-460): rows[:, :c] = prefix_rows, steps c + 1..n on the column order sigma [S, n];
    with `avoid`, before every step after the first free one a stream whose last row is avoided is
    dropped, and each pass chunk's survivors are renumbered (chunk start s - rng_off0[s]) before the next
    step's draws, whose stream offset is that rank; the last row is checked after the last step.
    A [G, m, n] complex, seeds [R, n], seed_row [S].  Returns (rows [S, n], alive [S] bool); a dropped
    stream keeps the rows drawn up to its drop and -1 after it."""
    A = _c128(A)
    if A.ndim == 2:
        A = A[None]
    dp = np.asarray(dp, dtype=np.int64).reshape(-1)
    S = dp.shape[0]
    sigma = np.asarray(sigma, dtype=np.int64).reshape(S, -1)
    n = sigma.shape[1]
    pre = np.asarray(prefix_rows, dtype=np.int64).reshape(S, -1)
    c0 = pre.shape[1]
    seeds = np.asarray(seeds, dtype=np.int64).reshape(-1, n)
    seed_row = np.asarray(seed_row, dtype=np.int64).reshape(-1)
    off0 = np.asarray(rng_off0, dtype=np.int64).reshape(-1)
    start = np.arange(S) - off0
    avoid_set = set(int(r) for r in avoid) if avoid is not None else None
    rows = np.full((S, n), -1, dtype=np.int64)
    rows[:, :c0] = pre
    alive = np.ones(S, dtype=bool)
    L = lib()
    for k in range(c0 + 1, n + 1):
        if avoid_set is not None and k > c0 + 1:
            alive = np.array([bool(alive[s]) and int(rows[s, k - 2]) not in avoid_set for s in range(S)])
        rank = np.zeros(S, dtype=np.int64)
        counts: dict = {}
        for s in range(S):
            if alive[s]:
                rank[s] = counts.get(int(start[s]), 0)
                counts[int(start[s])] = rank[s] + 1
        for s in range(S):
            if not alive[s]:
                continue
            u = L.oracle_uniform(int(seeds[seed_row[s], k - 1]), int(rank[s]))
            idx, _, _ = step(A[dp[s]], rows[s, :k - 1], sigma[s, :k], u, precision)
            rows[s, k - 1] = idx
    if avoid_set is not None and n > c0:
        alive = np.array([bool(alive[s]) and int(rows[s, n - 1]) not in avoid_set for s in range(S)])
    return rows, alive


def occupations(rows, m: int) -> np.ndarray:
    """[S, n] ordered output modes -> [S, m] int64 occupations."""
    rows = np.asarray(rows, dtype=np.int64)
    occ = np.zeros((rows.shape[0], m), dtype=np.int64)
    for j in range(rows.shape[1]):
        np.add.at(occ, (np.arange(rows.shape[0]), rows[:, j]), 1)
    return occ


# ---------------------------------------------------------------------------------------- exact references

def per_ryser(M) -> complex:
    """Permanent by Ryser's formula (an independent check; tests/clifford/check_cofactors.py:17-24)."""
    M = np.asarray(M, dtype=np.complex128)
    n = M.shape[0]
    if n == 0:
        return 1.0 + 0j
    tot = 0j
    for r in range(1, n + 1):
        for cols in itertools.combinations(range(n), r):
            tot += (-1) ** r * np.prod(M[:, list(cols)].sum(1))
    return tot * (-1) ** n


def ryser_cofactors(B) -> np.ndarray:
    B = np.asarray(B, dtype=np.complex128)
    K = B.shape[1]
    return np.array([per_ryser(np.delete(B, c, axis=1)) for c in range(K)])


def exact_distribution(U, in_modes) -> dict:
    """{occupation tuple: probability} of n photons in `in_modes` through U (all C(m+n-1, n) outcomes)."""
    U = np.asarray(U, dtype=np.complex128)
    m = U.shape[0]
    n = len(in_modes)
    A = U[:, list(in_modes)]
    s_fact = np.prod([math.factorial(c) for c in np.bincount(in_modes, minlength=m)])
    dist = {}
    for t in itertools.combinations_with_replacement(range(m), n):
        occ = np.bincount(t, minlength=m)
        p = abs(per_ryser(A[list(t), :])) ** 2 / (s_fact * np.prod([math.factorial(c) for c in occ]))
        dist[tuple(int(x) for x in occ)] = float(p)
    return dist


def imperfect_distribution(U, in_modes, eta: float, x: float) -> dict:
    """Exact law of lossy, x-model partially distinguishable photons: every photon independently lost
    (1 - eta), interfering (eta x) or alone (eta (1 - x)); the interfering ones follow the permanent law,
    each lone one lands in row r with probability |U[r, col]|^2, and the occupations add (the model of
    photonic_engines/imperfections.py, the reference's x_mixture in slos/species.py)."""
    U = np.asarray(U, dtype=np.complex128)
    m, n = U.shape[0], len(in_modes)
    dist: dict = {}
    for roles in itertools.product((0, 1, 2), repeat=n):        # 0 lost, 1 alone, 2 interfering
        p = 1.0
        for r in roles:
            p *= (1 - eta) if r == 0 else (eta * (1 - x) if r == 1 else eta * x)
        if p == 0.0:
            continue
        inter = [in_modes[j] for j in range(n) if roles[j] == 2]
        lone = [in_modes[j] for j in range(n) if roles[j] == 1]
        part = exact_distribution(U, inter) if inter else {tuple([0] * m): 1.0}
        for col in lone:
            w = np.abs(U[:, col]) ** 2
            new: dict = {}
            for k, q in part.items():
                for r_ in range(m):
                    kk = list(k)
                    kk[r_] += 1
                    new[tuple(kk)] = new.get(tuple(kk), 0.0) + q * w[r_]
            part = new
        for k, q in part.items():
            dist[k] = dist.get(k, 0.0) + p * q
    return dist


def tvd_and_floor(dist: dict, occ) -> tuple[float, float]:
    """Total-variation distance of the empirical histogram of `occ` [S, m] to `dist`, and its
    shot-noise level 0.5 sum sqrt(p (1 - p) / S) sqrt(2 / pi) (tests/clifford/check_sampler.py:59-60)."""
    occ = np.asarray(occ)
    S = occ.shape[0]
    emp: dict = {}
    for row in occ:
        key = tuple(int(x) for x in row)
        if key not in dist:
            raise AssertionError(f"impossible outcome {key}")
        emp[key] = emp.get(key, 0) + 1
    tvd = 0.5 * sum(abs(p - emp.get(k, 0) / S) for k, p in dist.items())
    floor = 0.5 * sum(math.sqrt(p * (1 - p) / S) for p in dist.values()) * math.sqrt(2 / math.pi)
    return tvd, floor


def haar_unitary(m: int, seed: int) -> np.ndarray:
    """Haar-random m x m unitary, complex128, deterministic in `seed` (tests/helpers.py:10-17:
    QR of a complex standard Gaussian from a seeded torch CPU generator, phase of diag(R) fixed)."""
    import torch
    g = torch.Generator().manual_seed(seed)
    z = torch.randn(m, m, generator=g, dtype=torch.float64) + 1j * torch.randn(m, m, generator=g, dtype=torch.float64)
    q, r = torch.linalg.qr(z)
    d = torch.diagonal(r)
    return (q * (d / d.abs()).unsqueeze(0)).numpy()


def chain_uniforms(seeds, seed_row, rng_off, steps: int) -> np.ndarray:
    """u [C, steps]: the uniform of chain c at step k is the draw kernel's uniform for seed
    seeds[seed_row[c], k] and stream offset rng_off[c]."""
    seeds = np.asarray(seeds, dtype=np.int64).reshape(-1, np.asarray(seeds).shape[-1])
    seed_row = np.asarray(seed_row, dtype=np.int64).reshape(-1)
    rng_off = np.asarray(rng_off, dtype=np.int64).reshape(-1)
    L = lib()
    out = np.empty((seed_row.shape[0], steps), dtype=np.float64)
    for c in range(seed_row.shape[0]):
        for k in range(steps):
            out[c, k] = L.oracle_uniform(int(seeds[seed_row[c], k]), int(rng_off[c]))
    return out
