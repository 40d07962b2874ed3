"""Typed torch-side wrappers of the two compute entry points of the CUDA library.

    chain(...)                 pe_fock_chain: whole Clifford & Clifford chains in one persistent launch
    laplace_cofactors_rows(..) pe_cofactors_rows: the cofactor step alone
                               (photonic_engines/clifford/cofactors_triton.py:509-530)
    pack_instances(...)        circuit input columns -> the column-major instance layout the chain reads

All tensors are CUDA tensors; launches go on torch's current stream of that device.
"""
from __future__ import annotations

import functools

import torch

from .. import _native as N


def pack_instances(U: torch.Tensor, in_modes) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    """U [B, m, m] (or [m, m]) and the n input modes -> (acol, inst_off, inst_m, inst_n).

    Instance b holds the n input columns U[b][:, in_modes] column-major: acol[b, j, rho] = U[b, rho, in_modes[j]],
    complex128, so that one input column is m contiguous complex values.
    """
    if U.dim() == 2:
        U = U[None]
    B, m, _ = U.shape
    idx = torch.as_tensor(list(in_modes), dtype=torch.int64, device=U.device)
    acol = U.to(torch.complex128)[:, :, idx].transpose(1, 2).contiguous()            # [B, n, m]
    n = idx.shape[0]
    dev = U.device
    inst_off = torch.arange(B, dtype=torch.int64, device=dev) * (n * m)
    inst_m = torch.full((B,), m, dtype=torch.int32, device=dev)
    inst_n = torch.full((B,), n, dtype=torch.int32, device=dev)
    return acol, inst_off, inst_m, inst_n


def pack_ragged(circuits) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    """Instances of different sizes: circuits = [(U_g [m_g, m_g], in_modes_g)] -> one flat acol buffer with
    per-instance offsets, modes and column counts (the many-instance batch)."""
    parts, off, ms, ns = [], [], [], []
    pos = 0
    dev = circuits[0][0].device
    for U, modes in circuits:
        idx = torch.as_tensor(list(modes), dtype=torch.int64, device=U.device)
        a = U.to(torch.complex128)[:, idx].transpose(0, 1).contiguous().reshape(-1)   # [n_g * m_g]
        parts.append(a)
        off.append(pos)
        ms.append(U.shape[0])
        ns.append(idx.shape[0])
        pos += a.shape[0]
    acol = torch.cat(parts)
    return (acol, torch.tensor(off, dtype=torch.int64, device=dev), torch.tensor(ms, dtype=torch.int32, device=dev),
            torch.tensor(ns, dtype=torch.int32, device=dev))


def _i64(t, dev):
    return None if t is None else torch.as_tensor(t, dtype=torch.int64, device=dev).contiguous()


def _seed_rows(seeds_t, seed_row_t):
    """seed_row indexes the rows of seeds: checked on the host before a launch reads seeds with it."""
    if seeds_t is None or seed_row_t is None or seed_row_t.numel() == 0:
        return
    lo, hi = int(seed_row_t.min()), int(seed_row_t.max())
    if lo < 0 or hi >= seeds_t.shape[0]:
        raise ValueError(f"seed_row: values in [0, {seeds_t.shape[0]}) expected (got {lo}..{hi})")


DEFAULT_BLOCK = 128          # the library's CTA size when the caller passes 0 (pe_fock_chain)


def default_tpl(n: int, precision: str) -> int:
    """Threads per Gray lane the library picks when the caller passes 0 (fock_api.cu default_tpl)."""
    kpm = next((k for k in (8, 16, 20, 24, 28, 32, 40, 48, 56, 64) if n <= k), 64)
    if kpm <= 8 or (precision != "compensated" and kpm == 20):
        return 1
    if precision == "compensated":
        return 2 if kpm <= 20 else 4
    return 2 if kpm <= 40 else 4


NCH_MAX = 512                # CTAs per stream at most
# split work items (streams x nch) per resident split CTA, at least; more for chains of 24+ photons, whose
# later steps have fewer live streams and far more terms (measured, FP64 ms: c4 n = 28 m = 784 200 shots
# 471 -> 379, n = 28 m = 56 256 shots 150 -> 124, n = 26 m = 52 512 shots 84 -> 76; n = 32 m = 64 32 shots
# 195 -> 204; for n = 20, m = 400, 100 shots the smaller fill stays faster, 2.6 against 3.3)
SPLIT_FILL = 6
SPLIT_FILL_LONG = 24

# Chains of at most this many photons run the FP64 kernels when the plain mixed form is asked for: their
# sweeps are too short for FP32 to pay (n = 6, m = 12, 10 000 shots: mixed 36.3 M against FP64 39.0 M
# samples/s on B200), and the mixed form returns the FP64 form's picks anyway.
MIXED_MIN_PHOTONS = 9


def effective_precision(precision: str, n: int) -> str:
    """The precision the kernels run for chains of n photons when `precision` is asked for."""
    return "f64" if precision == "mixed" and n < MIXED_MIN_PHOTONS else precision


@functools.lru_cache(maxsize=None)
def _split_slots(device_index: int, precision: str, n: int, block_threads: int, tpl: int) -> int:
    L = N.load()
    with torch.cuda.device(device_index):
        slots = int(L.pe_split_slots(N.PRECISIONS[precision], n, block_threads, tpl))
    N.check(min(slots, 0), "pe_split_slots")
    return slots


def split_plan(heavy_streams: int, n: int, device, block_threads: int = 0, tpl: int = 2, precision: str = "f64"):
    """(k_split, nch) for a batch whose long chains number `heavy_streams`, or None when one CTA per stream
    already fills the GPU several times over.  nch CTAs share every step k >= k_split of a stream.

    nch is a power of two (a step's Gray lanes come in powers of two, so any other count leaves lanes idle)
    with heavy_streams * nch at least SPLIT_FILL (24 photons and more: SPLIT_FILL_LONG) times the split
    kernel's resident CTAs (`pe_split_slots`), so that the last partial wave costs little; at most 512, and at most what leaves the last four steps split
    (2^(n-2) / (32 lanes)); of nch and 2 nch the one that fills its waves better (by more than 2 %) wins.  k_split is the first step with enough Gray terms (2^(k-2)) for every
    CTA to run several lanes.  The reference's single-sample path sizes a fixed lane grid instead
    (photonic_engines/clifford/single.py:22-82)."""
    if n < 8 or heavy_streams < 1:
        return None
    dev = torch.device(device)
    block = block_threads or DEFAULT_BLOCK
    tpl = tpl or default_tpl(n, precision)
    slots = _split_slots(dev.index if dev.index is not None else torch.cuda.current_device(), precision, n,
                         block, tpl)
    if heavy_streams >= 3 * slots:
        return None

    def fill(c):
        items = heavy_streams * c
        return items / (-(-items // slots) * slots)

    lanes = block // max(tpl, 1)
    # at most enough CTAs for the last four steps to be split (short chains: earlier steps stay whole)
    cap = max(1, min(NCH_MAX, (1 << (n - 2)) // (32 * lanes)))
    nch = 1
    waves = SPLIT_FILL_LONG if n >= 24 else SPLIT_FILL
    while nch < cap and heavy_streams * nch < waves * slots:
        nch *= 2
    if 2 * nch <= cap and fill(2 * nch) > fill(nch) + 0.02:
        nch *= 2
    if nch == 1:
        return None
    k = 2
    while k <= n and (1 << (k - 2)) < 4 * nch * lanes:
        k += 1
    return (k, nch) if k <= n else None


WARP_MAX_PHOTONS = 16


def use_warp_form(S: int, n: int, device) -> bool:
    """The warp-per-stream form for short chains: always up to 12 photons, up to 16 when the streams are
    many enough to fill the GPU's warps."""
    if n > WARP_MAX_PHOTONS:
        return False
    return n <= 12 or S >= 64 * torch.cuda.get_device_properties(device).multi_processor_count


# Length tiers of a ragged launch (lossy or partially distinguishable shots): the photon counts at which the
# longest-first queue is cut, so that every chain runs in the smallest kernel variant that holds it, and the
# count above which the few longest chains have their heavy steps split over several CTAs (one 26-photon
# survivor at m = 900 otherwise holds one CTA for longer than all the other chains of 10 000 shots take).
TIER_CUTS = (20, 16)
LONG_SPLIT_ABOVE = 24


def tier_plan(counts: dict, n_stride: int, precision: str, device) -> list:
    """The tiers of a ragged launch whose chains are queued longest first: counts {photons: chains} ->
    [(lo, hi, nk_max, mode, split)] over queue positions [lo, hi), chains of at most nk_max photons; mode 0
    one CTA per chain, 1 one warp per chain (the last tier, up to 16 photons, FP64 and mixed forms), 2 one
    CTA per chain with steps k_split.. spread over nch CTAs (split = (k_split, nch), the chains above
    LONG_SPLIT_ABOVE photons when they are too few to fill the GPU).  Empty counts give no tier."""
    bounds = [n_stride] + ([LONG_SPLIT_ABOVE] if n_stride > LONG_SPLIT_ABOVE else [])
    bounds += [c for c in TIER_CUTS if c < bounds[-1]] + [0]
    tiers, pos = [], 0
    for i in range(len(bounds) - 1):
        ks = [k for k, c in counts.items() if bounds[i + 1] < k <= bounds[i] and c > 0]
        if not ks:
            continue
        cnt, nk_max = sum(counts[k] for k in ks), max(ks)
        mode, split = 0, None
        if bounds[i + 1] == LONG_SPLIT_ABOVE:
            split = split_plan(cnt, nk_max, device, DEFAULT_BLOCK, default_tpl(nk_max, precision), precision)
            mode = 2 if split else 0
        elif bounds[i + 1] == 0 and precision != "compensated" and use_warp_form(cnt, nk_max, device):
            mode = 1
        tiers.append((pos, pos + cnt, nk_max, mode, split))
        pos += cnt
    return tiers


_SIDE_STREAMS: dict = {}


def _side_streams(dev, count: int) -> list:
    """Side streams of a device for concurrent tiers (made once, reused)."""
    key = dev.index if dev.index is not None else torch.cuda.current_device()
    have = _SIDE_STREAMS.setdefault(key, [])
    while len(have) < count:
        have.append(torch.cuda.Stream(dev))
    return have[:count]


def chain_tiers(acol: torch.Tensor, inst_off: torch.Tensor, inst_m: torch.Tensor, inst_n: torch.Tensor, dp, cols, nk,
                order, tiers, *, m_max: int, seeds, seed_row=None, rng_off=None, precision: str = "f64",
                check_status: bool = True) -> torch.Tensor:
    """Ragged chains (nk [C] photons, order [C] queue of chains longest first) in the length tiers of
    `tier_plan`, one launch per tier (pe_fock_chain_range / pe_fock_chain_range_split), the tiers on
    concurrent streams joined back into the current one.  Philox draws from seeds only.  Returns the
    ordered rows [C, n_stride] (entries past nk[c] untouched, zero)."""
    N.require_cuda(acol, "acol")
    dev = acol.device
    L = N.load()
    if precision not in N.PRECISIONS:
        raise ValueError(f"unknown precision {precision!r}: 'f64', 'mixed' or 'compensated'")
    dp, cols, order_t = _i64(dp, dev), _i64(cols, dev), _i64(order, dev)
    C, n_stride = cols.shape
    N.check_photons(n_stride, precision)
    nk_t = torch.as_tensor(nk, dtype=torch.int32, device=dev).contiguous()
    seeds_t = _i64(seeds, dev)
    if seeds_t.dim() == 1:
        seeds_t = seeds_t[None]
    if seeds_t.shape[-1] != n_stride:
        seeds_t = torch.nn.functional.pad(seeds_t, (0, n_stride - seeds_t.shape[-1])).contiguous()
    seed_row_t, rng_off_t = _i64(seed_row, dev), _i64(rng_off, dev)
    _seed_rows(seeds_t, seed_row_t)
    if not tiers or tiers[-1][1] != C or any(a[1] != b[0] for a, b in zip(tiers, tiers[1:])) or tiers[0][0] != 0:
        raise ValueError("tiers: consecutive queue ranges covering every chain expected")
    rows = torch.zeros(C, n_stride, dtype=torch.int64, device=dev)
    a = acol if acol.dtype == torch.float64 else torch.view_as_real(acol.contiguous())
    # every buffer a tier reads is made on the current stream before the side streams wait on it
    qr = torch.tensor([[lo, hi] for lo, hi, *_ in tiers], dtype=torch.int64, device=dev)
    wss = []
    for lo, hi, nk_max, mode, split in tiers:
        nb = L.pe_range_split_workspace_bytes(hi - lo, split[1]) if mode == 2 else L.pe_chain_workspace_bytes(C)
        wss.append(torch.zeros(int(nb), dtype=torch.uint8, device=dev))
    cur = torch.cuda.current_stream(dev)
    side = _side_streams(dev, len(tiers) - 1)
    for s_ in side:
        s_.wait_stream(cur)
    for i, (lo, hi, nk_max, mode, split) in enumerate(tiers):
        st = (cur if i == 0 else side[i - 1]).cuda_stream
        prec = effective_precision(precision, nk_max)
        common = (N.PRECISIONS[prec], N.ptr(a), N.ptr(inst_off), N.ptr(inst_m), N.ptr(inst_n), int(inst_off.shape[0]),
                  int(m_max), int(C), N.ptr(dp), N.ptr(nk_t), N.ptr(cols), int(n_stride), None, N.ptr(seeds_t),
                  N.ptr(seed_row_t), N.ptr(rng_off_t), N.ptr(order_t), N.ptr(rows), None, int(m_max), None,
                  int(m_max), N.ptr(wss[i]), int(wss[i].numel()))
        if mode == 2:
            rc = L.pe_fock_chain_range_split(*common, DEFAULT_BLOCK, default_tpl(nk_max, prec), N.ptr(qr[i]), int(nk_max),
                                             int(split[0]), int(split[1]), int(hi - lo), st)
            N.check(rc, "pe_fock_chain_range_split")
        else:
            rc = L.pe_fock_chain_range(*common, 0, 0, 0, N.ptr(qr[i]), int(nk_max), int(mode), st)
            N.check(rc, "pe_fock_chain_range")
    for s_ in side:
        cur.wait_stream(s_)
    if check_status:
        for ws in wss:
            st_, det = N.read_status(ws)
            if st_ != 0:
                raise N.NativeError(f"pe_fock_chain_range: device-side index error at stream {det} (status {st_})")
    return rows


def chain(acol: torch.Tensor, inst_off: torch.Tensor, inst_m: torch.Tensor, inst_n: torch.Tensor, dp, cols, *,
          m_max: int | None = None, nk=None, uniforms=None, seeds=None, seed_row=None, rng_off=None, order=None,
          want_occ: bool = True, occ_stride: int | None = None, want_marg: bool = False, precision: str = "f64",
          block_threads: int = 0, tpl: int = 0, grid_ctas: int = 0, check_status: bool = True, out=None,
          split=None, mode: str = "auto"):
    """Run the chains of S streams.  dp [S] instance per stream, cols [S, n_stride] input columns in chain order,
    nk [S] photons per stream (None: n_stride), uniforms [S, n_stride] (None: Philox from seeds [R, n_stride],
    seed_row [S], rng_off [S]).  Returns (rows [S, n_stride] int64, occ [S, occ_stride] or None,
    marg [S, n_stride, m_max] or None).  `out` may hold preallocated (rows, occ, marg) tensors.
    split: (k_split, nch) spreads every step k >= k_split over nch CTAs per stream (few-stream batches);
    None or False runs each stream in one CTA.  mode: "cta" (one CTA per stream), "warp" (one warp per
    stream, n_stride <= 16) or "auto" (warp form for short chains, see use_warp_form)."""
    N.require_cuda(acol, "acol")
    dev = acol.device
    L = N.load()
    if precision not in N.PRECISIONS:
        raise ValueError(f"unknown precision {precision!r}: 'f64', 'mixed' or 'compensated'")
    dp = _i64(dp, dev)
    cols = _i64(cols, dev)
    S, n_stride = cols.shape
    N.check_photons(n_stride, precision)
    precision = effective_precision(precision, n_stride)
    if m_max is None:
        m_max = int(inst_m.max().item())
    occ_stride = occ_stride or m_max
    nk_t = None if nk is None else torch.as_tensor(nk, dtype=torch.int32, device=dev).contiguous()
    u_t = None if uniforms is None else torch.as_tensor(uniforms, dtype=torch.float64, device=dev).contiguous()
    seeds_t = _i64(seeds, dev)
    if u_t is None and seeds_t is None:
        raise ValueError("either uniforms or seeds")
    if seeds_t is not None and seeds_t.dim() == 1:
        seeds_t = seeds_t[None]
    if seeds_t is not None and seeds_t.shape[-1] != n_stride:
        seeds_t = torch.nn.functional.pad(seeds_t, (0, n_stride - seeds_t.shape[-1])).contiguous()
    # converted tensors stay referenced until the launch is queued (temporaries freed inside the argument
    # list would let the next conversion reuse their memory)
    seed_row_t, rng_off_t, order_t = _i64(seed_row, dev), _i64(rng_off, dev), _i64(order, dev)
    _seed_rows(seeds_t, seed_row_t)
    if out is not None:
        rows, occ, marg = out
    else:
        rows = torch.zeros(S, n_stride, dtype=torch.int64, device=dev)
        occ = torch.empty(S, occ_stride, dtype=torch.int64, device=dev) if want_occ else None
        marg = torch.zeros(S, n_stride, m_max, dtype=torch.float64, device=dev) if want_marg else None
    a = acol if acol.dtype == torch.float64 else torch.view_as_real(acol.contiguous())
    common = (N.PRECISIONS[precision], N.ptr(a), N.ptr(inst_off), N.ptr(inst_m), N.ptr(inst_n), int(inst_off.shape[0]),
              int(m_max), int(S), N.ptr(dp), N.ptr(nk_t), N.ptr(cols), int(n_stride), N.ptr(u_t), N.ptr(seeds_t),
              N.ptr(seed_row_t), N.ptr(rng_off_t), N.ptr(order_t), N.ptr(rows), N.ptr(occ),
              int(occ_stride), N.ptr(marg), int(m_max))
    if mode not in ("auto", "cta", "warp"):
        raise ValueError(f"unknown mode {mode!r}: 'auto', 'cta' or 'warp'")
    warp = (mode == "warp") or (mode == "auto" and not split and precision != "compensated"
                                and use_warp_form(S, n_stride, dev))
    if warp:
        ws = N.workspace(dev)
        rc = L.pe_fock_chain_warp(*common, N.ptr(ws), int(ws.numel()), int(tpl if tpl in (1, 2) else 0),
                                  int(grid_ctas), N.stream_handle(dev))
        N.check(rc, "pe_fock_chain_warp")
    elif split:
        k_split, nch = split
        ws = torch.empty(int(L.pe_chain_split_workspace_bytes(S, nch)), dtype=torch.uint8, device=dev)
        rc = L.pe_fock_chain_split(*common, int(k_split), int(nch), N.ptr(ws), int(ws.numel()), int(block_threads),
                                   int(tpl), N.stream_handle(dev))
        N.check(rc, "pe_fock_chain_split")
    else:
        ws = N.workspace(dev)
        rc = L.pe_fock_chain(*common, N.ptr(ws), int(ws.numel()), int(block_threads), int(tpl), int(grid_ctas),
                             N.stream_handle(dev))
        N.check(rc, "pe_fock_chain")
    if check_status:
        st, det = N.read_status(ws)
        if st != 0:
            raise N.NativeError(f"pe_fock_chain: device-side index error at stream {det} (status {st})")
    return rows, occ, marg


def chain_adaptive(acol: torch.Tensor, inst_off: torch.Tensor, inst_m: torch.Tensor, inst_n: torch.Tensor, dp, cols,
                   rows: torch.Tensor, n_prefix: int, *, m_max: int | None = None, avoid=None, uniforms=None,
                   seeds=None, seed_row=None, rng_off=None, precision: str = "f64", block_threads: int = 0,
                   tpl: int = 0, split=None, mode: str = "auto", check_status: bool = True):
    """Adaptive chains (pe_fock_chain_adaptive): rows [S, n] int64 holds the forced prefix in its first
    n_prefix columns and receives the rest; avoid: bool / uint8 [m_max] mask of avoided modes or None.
    Every stream has n = cols.shape[1] photons.  Returns (rows, occ [S, m_max], alive [S] bool)."""
    N.require_cuda(acol, "acol")
    dev = acol.device
    L = N.load()
    if precision not in N.PRECISIONS:
        raise ValueError(f"unknown precision {precision!r}: 'f64', 'mixed' or 'compensated'")
    dp = _i64(dp, dev)
    cols = _i64(cols, dev)
    S, n = cols.shape
    N.check_photons(n, precision)
    precision = effective_precision(precision, n)
    if m_max is None:
        m_max = int(inst_m.max().item())
    u_t = None if uniforms is None else torch.as_tensor(uniforms, dtype=torch.float64, device=dev).contiguous()
    seeds_t = _i64(seeds, dev)
    if u_t is None and seeds_t is None:
        raise ValueError("either uniforms or seeds")
    if seeds_t is not None and seeds_t.dim() == 1:
        seeds_t = seeds_t[None]
    seed_row_t, rng_off_t = _i64(seed_row, dev), _i64(rng_off, dev)
    _seed_rows(seeds_t, seed_row_t)
    av = None
    if avoid is not None:
        av = torch.as_tensor(avoid, device=dev).to(torch.uint8).contiguous()
        if av.shape != (m_max,):
            raise ValueError(f"avoid: a mask over the {m_max} output modes")
    alive = torch.ones(S, dtype=torch.uint8, device=dev)
    occ = torch.zeros(S, m_max, dtype=torch.int64, device=dev)
    if mode not in ("auto", "cta", "warp"):
        raise ValueError(f"unknown mode {mode!r}: 'auto', 'cta' or 'warp'")
    warp = (mode == "warp") or (mode == "auto" and not split and precision != "compensated"
                                and use_warp_form(S, n, dev))
    k_split, nch = (0, 0) if (warp or not split) else split
    ws = torch.empty(int(L.pe_adaptive_workspace_bytes(S, nch)), dtype=torch.uint8, device=dev)
    a = acol if acol.dtype == torch.float64 else torch.view_as_real(acol.contiguous())
    rc = L.pe_fock_chain_adaptive(N.PRECISIONS[precision], N.ptr(a), N.ptr(inst_off), N.ptr(inst_m), N.ptr(inst_n),
                                  int(inst_off.shape[0]), int(m_max), int(S), N.ptr(dp), N.ptr(cols), int(n),
                                  N.ptr(u_t), N.ptr(seeds_t), N.ptr(seed_row_t), N.ptr(rng_off_t),
                                  N.ptr(rows), int(n_prefix), N.ptr(av), N.ptr(alive), N.ptr(occ), int(m_max),
                                  int(k_split), int(nch), N.ptr(ws), int(ws.numel()), int(block_threads),
                                  int(tpl if (not warp or tpl in (1, 2)) else 0), 1 if warp else 0,
                                  N.stream_handle(dev))
    N.check(rc, "pe_fock_chain_adaptive")
    if check_status:
        st, det = N.read_status(ws)
        if st != 0:
            raise N.NativeError(f"pe_fock_chain_adaptive: device-side index error at stream {det} (status {st})")
    return rows, occ, alive.bool()


def laplace_cofactors_rows(A: torch.Tensor, rows: torch.Tensor, precision: str = "f64", block_threads: int = 0,
                           tpl: int = 0) -> torch.Tensor:
    """P [S, K] with P[s, c] = per(A[s][rows[s]] without column c); A [S, m, K] complex128, rows [S, K - 1]
    (repeats allowed).  Same contract as the reference's laplace_cofactors_rows."""
    N.require_cuda(A, "A")
    S, m, K = A.shape
    N.check_photons(K, precision, "columns")
    dev = A.device
    A2 = torch.view_as_real(A.to(torch.complex128).contiguous())
    rows = torch.as_tensor(rows, dtype=torch.int64, device=dev).reshape(S, K - 1).contiguous()
    P = torch.empty(S, K, dtype=torch.complex128, device=dev)
    ws = N.workspace(dev)
    rc = N.load().pe_cofactors_rows(N.PRECISIONS[precision], N.ptr(A2), N.ptr(rows) if K > 1 else None, int(S), int(m),
                                    int(K), N.ptr(torch.view_as_real(P)), N.ptr(ws), int(ws.numel()), int(block_threads),
                                    int(tpl), N.stream_handle(dev))
    N.check(rc, "pe_cofactors_rows")
    st, det = N.read_status(ws)
    if st != 0:
        raise N.NativeError(f"pe_cofactors_rows: device-side index error at block {det}")
    return P
