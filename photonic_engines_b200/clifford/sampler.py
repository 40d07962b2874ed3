"""Host orchestration of the exact Clifford & Clifford Fock sampler on B200.

`fock_sample(U, in_modes, shots, generator, loss=, indist=, ...)` keeps the reference's signature,
argument meaning, stream layout (row s = b * shots + shot), error behaviour and generator consumption
(photonic_engines/clifford/sampler.py:57-225), so that a seeded generator gives the reference's samples:

  * sigma = argsort(rand(S, n)) and the per-step seeds randint(0, 2^31 - 1, (n,)) per lockstep pass of at
    most `max_streams` streams (sampler.py:407, 411), in the reference's pass order;
  * the per-step uniforms are the reference's Philox draws, made inside the kernel;
  * loss / partial distinguishability: the shots are partitioned on the host generator and grouped by
    surviving column set and count exactly as the reference groups them (sampler.py:183-215); singleton
    photons are routed classically on the host.

What differs is the execution: every chain of every pass runs in ONE launch of the persistent chain kernel
(no per-step launches, no per-pass copies of U's columns, no host synchronisation inside the chain); a
ragged call (loss, partial distinguishability) runs one launch per length tier instead, on concurrent
streams, each tier in the smallest kernel variant that holds its chains and its few longest chains with
their heavy steps split over several CTAs (kernels.tier_plan).
"""
from __future__ import annotations

import time as _time
from dataclasses import dataclass

import torch

from .. import _native as N
from ..imperfections import as_model, draw_fates, group_fates, route_lone_photons
from .kernels import chain, chain_adaptive, chain_tiers, default_tpl, pack_instances, split_plan, tier_plan
from .prefix import prefix_order

BACKENDS = ("b200", "triton", "cuda", "exq")
ALGOS = ("auto", "2018", "2020", "input", "percof")


def _draw_device(generator, dev):
    return generator.device if generator is not None else dev


def _cpu_generator(generator):
    """The host generator of the partition draws: `generator` itself when it lives on the CPU, else a CPU
    generator seeded by one randint from it (sampler.py:218-225)."""
    if generator is None or generator.device.type == "cpu":
        return generator
    seed = int(torch.randint(0, 2 ** 31 - 1, (1,), generator=generator, device=generator.device).item())
    return torch.Generator().manual_seed(seed)


def _pass_draws(S: int, k: int, generator, dev, max_streams: int):
    """sigma [S, k] and per-chunk seeds for one lockstep pass of S streams, drawn chunk by chunk as the
    reference's `_sample_streams` draws them.  Returns (sigma, seeds [C, k], chunk index [S], offset [S])."""
    gdev = _draw_device(generator, dev)
    sig, seeds, chunk, off = [], [], [], []
    for ci, c0 in enumerate(range(0, S, max_streams)):
        Sc = min(max_streams, S - c0)
        sig.append(torch.argsort(torch.rand(Sc, k, generator=generator, device=gdev), dim=1).to(dev))
        seeds.append(torch.randint(0, 2 ** 31 - 1, (k,), generator=generator, device=gdev).to(dev))
        chunk.append(torch.full((Sc,), ci, dtype=torch.int64, device=dev))
        off.append(torch.arange(Sc, dtype=torch.int64, device=dev))
    if not sig:
        z = torch.zeros(0, k, dtype=torch.int64, device=dev)
        return z, torch.zeros(0, k, dtype=torch.int64, device=dev), z[:, 0], z[:, 0]
    return torch.cat(sig), torch.stack(seeds), torch.cat(chunk), torch.cat(off)


def sample_chains(U, in_modes, sigma, *, uniforms=None, seeds=None, seed_row=None, rng_off=None, dp=None,
                  precision: str = "f64", want_marg: bool = False, block_threads: int = 0, tpl: int = 0,
                  grid_ctas: int = 0, split=False, mode: str = "auto"):
    """The chains of S streams with a GIVEN column order: sigma [S, n] (indices into in_modes), per-step
    uniforms [S, n] (or the reference's Philox draws from seeds [n] / [R, n]).  dp [S]: circuit of each stream
    (default: all circuit 0 when U is [m, m], else b * shots layout is the caller's).
    split: False (one CTA per stream), None (spread heavy steps over several CTAs when the streams are too
    few to fill the GPU) or an explicit (k_split, nch).  mode: "auto" | "cta" | "warp" (kernels.chain).
    Returns dict(rows [S, n] ordered output modes, occ [S, m], marg [S, n, m] or None)."""
    N.require_cuda(U, "U")
    if U.dim() == 2:
        U = U[None]
    dev = U.device
    sigma = torch.as_tensor(sigma, dtype=torch.int64, device=dev)
    S, n = sigma.shape
    if dp is None:
        dp = torch.zeros(S, dtype=torch.int64, device=dev)
    acol, inst_off, inst_m, inst_n = pack_instances(U, in_modes)
    if split is None:
        split = split_plan(S, n, dev, block_threads, tpl or default_tpl(n, precision), precision)
    rows, occ, marg = chain(acol, inst_off, inst_m, inst_n, dp, sigma, uniforms=uniforms, seeds=seeds,
                            seed_row=seed_row, rng_off=rng_off, want_occ=True, want_marg=want_marg,
                            precision=precision, block_threads=block_threads, tpl=tpl, grid_ctas=grid_ctas,
                            split=split, mode=mode)
    return {"rows": rows, "occ": occ, "marg": marg}


def fock_sample(U, in_modes, shots, generator=None, algo="auto", multi_min_k1=10, max_lanes=1 << 16,
                target_total_lanes=1 << 17, backend="b200", single_lanes=1 << 15, max_streams=1 << 18, loss=None,
                indist=None, prefix=None, avoid=None, keep_ids=False, stats=None, *, precision="f64", uniforms=None,
                block_threads=0, tpl=0):
    """Exact samples: occupations [S, m] int64 on U's device, S = B * shots (row s = b * shots + shot).

    U [B, m, m] or [m, m] complex (CUDA); in_modes the n input modes (repeats allowed); shots an int or an int
    tensor [B] of per-circuit counts (lossless only); generator a torch.Generator (on U's device, or on the
    CPU: its draws are then made on the host and copied).  loss: uniform transmission eta; indist: partial
    distinguishability (x-model float or `imperfections.Distinguishability`).  backend: "b200" (this library;
    "triton" and "cuda" are accepted and run the same kernels); algo: any of the reference's algorithms —
    they all draw the same chain, which is what runs.  multi_min_k1 / max_lanes / target_total_lanes /
    single_lanes are the reference's kernel tuning knobs and have no effect here.
    precision: "f64" (complex FP64, the drop-in), "mixed" (FP32 Gray blocks with FP64 cross-block sums,
    marginals and CDF; ~1e-5 marginals at 20 photons; chains of at most 8 photons run the FP64 kernels, which
    are faster there) or "compensated" (double-float FP32 Gray blocks: FP64-level marginals); every form
    returns the FP64 form's samples.  uniforms: optional float64 [S, n] per-step uniforms replacing the Philox draws
    (lossless only).  stats: receives "passes" = [(k, streams, seconds)] — all passes run in one launch (one
    per length tier when ragged), so every entry carries the launches' time — and "fused_seconds".
    prefix (adaptive sampling, lossless only): the output modes the FIRST c photons of every chain are forced
    onto — a list of c modes shared by all circuits, or an int tensor [B, c]; the column set of those c steps
    is drawn from its posterior |per(A[prefix, T])|^2 (`prefix.prefix_columns_many`) and the chain runs steps
    c + 1..n; the occupations include the prefix.  avoid: output modes no photon after the prefix may reach;
    a stream is dropped as soon as one does, and only the survivors are returned ([S', m]; with keep_ids=True
    the pair (occupations, surviving stream ids)).  Both as the reference's sampler.py:26-39, 391-460.
    """
    d = as_model(indist)
    if prefix is not None:
        prefix = torch.as_tensor(prefix, dtype=torch.int64)
        if prefix.dim() == 2 and prefix.shape[0] == 1 and U.dim() == 2:
            prefix = prefix[0]
        if prefix.numel() == 0:
            prefix = None
    avoid = [int(r) for r in avoid] if avoid is not None and len(avoid) else None
    if prefix is not None or avoid is not None:
        if backend == "exq" or d is not None or not (loss is None or float(loss) >= 1.0):
            raise NotImplementedError("prefix / avoid: lossless, indistinguishable photons only")
        nb = U.shape[0] if U.dim() == 3 else 1
        if prefix is not None:
            if prefix.dim() == 2 and prefix.shape[0] != nb:
                raise ValueError(f"prefix [{prefix.shape[0]}, r]: one row per circuit ({nb})")
            if (prefix.dim() > 2 or prefix.shape[-1] > len(in_modes) or bool((prefix < 0).any())
                    or bool((prefix >= U.shape[-2]).any())):
                raise ValueError(f"prefix: at most n = {len(in_modes)} output modes of the circuit")
        if avoid is not None and any(not 0 <= r < U.shape[-2] for r in avoid):
            raise ValueError(f"avoid {avoid}: output modes of the circuit")
    if backend not in BACKENDS:
        raise ValueError(f'unknown backend {backend!r} for a Fock input: "b200", "triton", "cuda" or "exq" '
                         f'("torch" exists on the emitter sampler only)')
    if algo not in ALGOS:
        raise ValueError(f'unknown algo {algo!r}: "auto", "2018", "2020", "input" or "percof"')
    if algo == "input" and backend == "cuda":
        raise NotImplementedError('algo="input": Triton kernel only (backend="triton")')
    if backend == "exq":
        raise NotImplementedError("backend 'exq' (the exqalibur 2017 benchmark port) is not part of this library")
    if precision not in N.PRECISIONS:
        raise ValueError(f"unknown precision {precision!r}: 'f64' or 'mixed'")
    N.require_cuda(U, "U")
    if U.dim() == 2:
        U = U[None]
    Bn, m, _ = U.shape
    n = len(in_modes)
    dev = U.device
    N.check_photons(n, precision, "photons")
    if any(not 0 <= int(j) < m for j in in_modes):
        raise ValueError(f"in_modes {list(in_modes)}: input modes of the circuit")
    lossless = loss is None or float(loss) >= 1.0
    reps = None
    if isinstance(shots, torch.Tensor):
        reps = shots.to(dev, torch.int64).reshape(-1)
        if reps.shape[0] != Bn or bool((reps < 0).any()):
            raise ValueError(f"shots [{reps.shape[0]}]: one non-negative count per circuit ({Bn})")
        if d is not None or not lossless:
            raise NotImplementedError("per-circuit shots: lossless, indistinguishable photons only")
        S = int(reps.sum())
    else:
        S = Bn * int(shots)
    dp_all = torch.arange(Bn, device=dev, dtype=torch.int64).repeat_interleave(reps if reps is not None else int(shots))
    occ = torch.zeros(S, m, dtype=torch.int64, device=dev)
    if n == 0 or S == 0:
        return (occ, torch.arange(S, device=dev, dtype=torch.int64)) if keep_ids else occ
    if uniforms is not None and not (lossless and d is None):
        raise NotImplementedError("uniforms=: lossless, indistinguishable photons only")
    if prefix is not None or avoid is not None:
        return _adaptive(U, in_modes, S, dp_all, generator, max_streams, prefix, avoid, keep_ids, stats,
                         precision, uniforms, block_threads, tpl)
    plan = plan_chains(U, in_modes, S, dp_all, generator, loss, d, max_streams)
    acol, inst_off, inst_m, inst_n = pack_instances(U, in_modes)
    t0 = None
    if stats is not None:
        torch.cuda.synchronize(dev)
        t0 = _time.perf_counter()
    rows = None
    direct = plan.out_row is None
    if plan.C > 0:
        u = None if uniforms is None else torch.as_tensor(uniforms, dtype=torch.float64, device=dev)
        tiers = []
        if plan.nk is not None and not direct and u is None and not block_threads and not tpl:
            counts: dict = {}
            for k, cnt in plan.passes:
                counts[k] = counts.get(k, 0) + cnt
            tiers = tier_plan(counts, n, precision, dev)
        if len(tiers) > 1 or (tiers and tiers[0][3] == 2):     # ragged: every length in its own tier
            rows = chain_tiers(acol, inst_off, inst_m, inst_n, plan.dp, plan.cols, plan.nk, plan.order, tiers,
                               m_max=m, seeds=plan.seeds, seed_row=plan.seed_row, rng_off=plan.rng_off,
                               precision=precision)
        else:
            heavy = plan.C if plan.nk is None else int((plan.nk >= 8).sum())
            rows, occ_k, _ = chain(acol, inst_off, inst_m, inst_n, plan.dp, plan.cols, m_max=m, nk=plan.nk, uniforms=u,
                                   seeds=plan.seeds, seed_row=plan.seed_row, rng_off=plan.rng_off, order=plan.order,
                                   want_occ=direct, precision=precision, block_threads=block_threads, tpl=tpl,
                                   split=split_plan(heavy, n, dev, block_threads,
                                                    tpl or default_tpl(n, precision), precision))
            if direct:
                occ = occ_k
    if stats is not None:
        torch.cuda.synchronize(dev)
        stats["fused_seconds"] = _time.perf_counter() - t0
        for k, cnt in plan.passes:
            stats.setdefault("passes", []).append((k, cnt, stats["fused_seconds"]))
    if not direct:
        occ = assemble_occupations(plan, rows, m)
    return (occ, torch.arange(S, device=dev, dtype=torch.int64)) if keep_ids else occ


def _adaptive(U, in_modes, S, dp_all, generator, max_streams, prefix, avoid, keep_ids, stats, precision, uniforms,
              block_threads, tpl):
    """fock_sample with a forced prefix and / or avoided modes (sampler.py:391-460 with prefix / avoid):
    per pass chunk of max_streams streams the column order (prefix_order for a prefix, else argsort(rand))
    and the step seeds, drawn as the reference draws them; then every chunk's chains in one call of the
    adaptive chain kernel (one launch per step with avoid, the survivors renumbered on the device)."""
    dev = U.device
    n = len(in_modes)
    m = U.shape[1]
    c0 = 0 if prefix is None else prefix.shape[-1]
    gdev = _draw_device(generator, dev)
    A = U[:, :, list(in_modes)].to(torch.complex128)
    sig, seeds, chunk, off = [], [], [], []
    for ci, s0 in enumerate(range(0, S, max_streams)):
        dpc = dp_all[s0:s0 + max_streams]
        Sc = dpc.shape[0]
        if c0:
            sig.append(prefix_order(A, dpc, n, prefix.to(dev), generator).to(dev))
        else:
            sig.append(torch.argsort(torch.rand(Sc, n, generator=generator, device=gdev), dim=1).to(dev))
        seeds.append(torch.randint(0, 2 ** 31 - 1, (n,), generator=generator, device=gdev).to(dev))
        chunk.append(torch.full((Sc,), ci, dtype=torch.int64, device=dev))
        off.append(torch.arange(Sc, dtype=torch.int64, device=dev))
    rows = torch.zeros(S, n, dtype=torch.int64, device=dev)
    if c0:
        pre = prefix.to(dev)
        rows[:, :c0] = pre[dp_all] if pre.dim() == 2 else pre
    mask = None
    if avoid is not None:
        mask = torch.zeros(m, dtype=torch.uint8, device=dev)
        mask[avoid] = 1
    acol, inst_off, inst_m, inst_n = pack_instances(U, in_modes)
    u = None if uniforms is None else torch.as_tensor(uniforms, dtype=torch.float64, device=dev)
    t0 = None
    if stats is not None:
        torch.cuda.synchronize(dev)
        t0 = _time.perf_counter()
    _, occ, alive = chain_adaptive(acol, inst_off, inst_m, inst_n, dp_all, torch.cat(sig), rows, c0, m_max=m,
                                   avoid=mask, uniforms=u, seeds=torch.stack(seeds), seed_row=torch.cat(chunk),
                                   rng_off=torch.cat(off), precision=precision, block_threads=block_threads, tpl=tpl,
                                   split=split_plan(S, n, dev, block_threads,
                                                    tpl or default_tpl(n, precision), precision))
    if stats is not None:
        torch.cuda.synchronize(dev)
        stats["fused_seconds"] = _time.perf_counter() - t0
        stats.setdefault("passes", []).append((n, S, stats["fused_seconds"]))
    if avoid is None:
        return (occ, torch.arange(S, device=dev, dtype=torch.int64)) if keep_ids else occ
    return (occ[alive], torch.nonzero(alive)[:, 0]) if keep_ids else occ[alive]


@dataclass
class ChainPlan:
    """Every chain of one `fock_sample` call, in the layout of the chain kernel.

    C chains; dp [C] circuit, cols [C, n] input columns in chain order (indices into in_modes), nk [C] photons
    (None: all n), seeds [R, n] per-pass-chunk step seeds, seed_row [C] / rng_off [C] the chunk and the local
    stream index of each chain, out_row [C] the output row of each chain (None: chain c is row c), order [C]
    the processing order, single_ids / single_rows the host-routed singleton photons, passes [(k, streams)].
    """
    S: int
    n: int
    C: int
    dp: torch.Tensor
    cols: torch.Tensor
    nk: torch.Tensor | None
    seeds: torch.Tensor
    seed_row: torch.Tensor
    rng_off: torch.Tensor
    out_row: torch.Tensor | None
    order: torch.Tensor | None
    single_ids: torch.Tensor | None
    single_rows: torch.Tensor | None
    passes: list


def plan_chains(U, in_modes, S: int, dp_all, generator, loss, indist, max_streams: int,
                _force_general: bool = False) -> ChainPlan:
    """The chains of a call and every host-side draw, consuming `generator` as the reference does
    (sampler.py:146-215): lossless -> one pass of S streams; otherwise the partition on the host generator,
    one pass per surviving count k over the distinct column sets, singletons routed classically last."""
    if U.dim() == 2:
        U = U[None]
    dev = U.device
    n = len(in_modes)
    d = as_model(indist)
    lossless = loss is None or float(loss) >= 1.0
    if lossless and d is None:
        sig, seeds, chunk, off = _pass_draws(S, n, generator, dev, max_streams)
        return ChainPlan(S, n, S, dp_all, sig, None, seeds, chunk, off, None, None, None, None, [(n, S)])
    gen = _cpu_generator(generator)
    if d is None and len(set(int(j) for j in in_modes)) == n and not _force_general:
        return _plan_loss_only(U, in_modes, S, dp_all, generator, gen, loss, max_streams)
    by_cols: dict = {}                       # column tuple -> [stream ids]
    rep_sub: dict = {}                       # column tuple -> photon indices (columns of the packed instance)
    single_ids, single_cols = [], []
    for subsets, singles, ids in group_fates(draw_fates(n, S, loss, d, generator=gen)):
        for sub in subsets:
            cols = tuple(int(in_modes[j]) for j in sub)
            if len(cols) == 1:
                single_ids.append(ids)
                single_cols.append(torch.full_like(ids, cols[0]))
            else:
                by_cols.setdefault(cols, []).append(ids)
                rep_sub.setdefault(cols, list(sub))
        for j in singles:
            single_ids.append(ids)
            single_cols.append(torch.full_like(ids, int(in_modes[j])))
    by_k: dict = {}
    for cols, ids_l in by_cols.items():
        by_k.setdefault(len(cols), []).append((cols, torch.cat(ids_l)))
    ch_dp, ch_cols, ch_nk, ch_row, ch_off, ch_out, all_seeds, passes = [], [], [], [], [], [], [], []
    n_rows = 0
    for k, groups in by_k.items():
        ids = torch.cat([g for _, g in groups])
        gidx = torch.cat([torch.full((g.shape[0],), gi, dtype=torch.int64) for gi, (_, g) in enumerate(groups)])
        subs = torch.tensor([rep_sub[c] for c, _ in groups], dtype=torch.int64, device=dev)        # [G, k]
        sig, seeds, chunk, off = _pass_draws(ids.shape[0], k, generator, dev, max_streams)
        ch_dp.append(dp_all[ids.to(dev)])
        ch_cols.append(torch.nn.functional.pad(torch.gather(subs[gidx.to(dev)], 1, sig), (0, n - k)))
        ch_nk.append(torch.full((ids.shape[0],), k, dtype=torch.int32, device=dev))
        ch_row.append(chunk + n_rows)
        ch_off.append(off)
        ch_out.append(ids.to(dev))
        all_seeds.append(torch.nn.functional.pad(seeds, (0, n - k)))
        n_rows += seeds.shape[0]
        passes.append((k, int(ids.shape[0])))
    s_ids = s_rows = None
    if single_ids:                           # host draws after every pass has drawn (the reference's order)
        s_ids = torch.cat(single_ids).to(dev)
        s_rows = route_lone_photons(U, dp_all[s_ids].cpu(), torch.cat(single_cols), generator=gen).to(dev)
    if not ch_dp:
        z = torch.zeros(0, dtype=torch.int64, device=dev)
        return ChainPlan(S, n, 0, z, z.reshape(0, n), z.to(torch.int32), z.reshape(0, n), z, z, z, z, s_ids, s_rows, [])
    nk = torch.cat(ch_nk)
    order = torch.argsort(nk.to(torch.int64), descending=True, stable=True)       # longest chains first
    return ChainPlan(S, n, int(nk.shape[0]), torch.cat(ch_dp), torch.cat(ch_cols), nk, torch.cat(all_seeds),
                     torch.cat(ch_row), torch.cat(ch_off), torch.cat(ch_out), order, s_ids, s_rows, passes)


def _plan_loss_only(U, in_modes, S, dp_all, generator, gen, loss, max_streams) -> ChainPlan:
    """plan_chains for uniform loss with distinct input modes, in tensor ops: the same role draws, passes,
    stream order, per-pass draws and classical routing as the general loop.  A stream's group is its row of
    roles among torch.unique's sorted rows; every group is one column set (its surviving photons), so the
    passes are the groups' photon counts in order of first appearance, and within a pass the groups in
    sorted order, each group's streams in ascending order; one-photon groups are routed classically."""
    dev = U.device
    n = len(in_modes)
    fates = draw_fates(n, S, loss, None, generator=gen)
    # rows hold LOST or species 0 only, so their lexicographic order (the grouping order) is the order of
    # the survival bitmask with photon 0 as the most significant bit: a 1-D unique gives the same groups
    weights = torch.tensor([1 << (n - 1 - j) for j in range(n)], dtype=torch.int64)
    mask = ((fates == 1).to(torch.int64) * weights).sum(1)
    umask, inv = torch.unique(mask, return_inverse=True)
    kept = ((umask[:, None] // weights[None, :]) % 2).bool()            # [G, n] surviving photons
    kg = kept.sum(1)                                                     # photons per group
    G = int(umask.shape[0])
    multi = torch.nonzero(kg >= 2)[:, 0]
    ks = []
    for k in kg[multi].tolist():                                         # passes: first appearance
        if k not in ks:
            ks.append(k)
    rank = torch.full((n + 1,), len(ks), dtype=torch.int64)
    for r_, k in enumerate(ks):
        rank[k] = r_
    passes, tabs = [], []
    if ks:
        key = rank[kg[inv]] * G + inv                                    # pass, then group; streams stable
        key[kg[inv] < 2] = len(ks) * G + G                               # not in a pass
        order_s = torch.sort(key, stable=True).indices
        skey = key[order_s]
        # the host side of every pass (no generator use): its streams in order and each stream's photons
        for r_, k in enumerate(ks):
            sel = order_s[(skey >= r_ * G) & (skey < (r_ + 1) * G)]     # streams of this pass, in order
            groups_k, gidx = torch.unique_consecutive(inv[sel], return_inverse=True)
            subs = torch.nonzero(kept[groups_k])[:, 1].reshape(-1, k)    # [groups, k] photon ids
            tab = torch.zeros(sel.shape[0], n + 2, dtype=torch.int64)   # photons | stream id | k
            tab[:, :k] = subs[gidx]
            tab[:, n] = sel
            tab[:, n + 1] = k
            tabs.append(tab)
            passes.append((k, int(sel.shape[0])))
    s_ids = s_rows = None
    one = kg[inv] == 1
    C = sum(c for _, c in passes)
    if C:
        # the pass draws, pass by pass and chunk by chunk in the reference's order, straight into device
        # buffers; then the host tables in one copy
        gdev = _draw_device(generator, dev)
        R = sum(-(-c // max_streams) for _, c in passes)
        sig = torch.zeros(C, n, dtype=torch.int64, device=dev)
        seeds = torch.zeros(R, n, dtype=torch.int64, device=dev)
        rowoff = torch.empty(C, 2, dtype=torch.int64)                    # seed row | offset in the chunk
        c0 = r0 = 0
        for k, cnt in passes:
            for s0 in range(0, cnt, max_streams):
                Sc = min(max_streams, cnt - s0)
                sig[c0 + s0:c0 + s0 + Sc, :k] = torch.argsort(torch.rand(Sc, k, generator=generator, device=gdev),
                                                              dim=1)
                seeds[r0, :k] = torch.randint(0, 2 ** 31 - 1, (k,), generator=generator, device=gdev)
                rowoff[c0 + s0:c0 + s0 + Sc, 0] = r0
                rowoff[c0 + s0:c0 + s0 + Sc, 1] = torch.arange(Sc)
                r0 += 1
            c0 += cnt
        host = torch.cat([torch.cat(tabs), rowoff], dim=1).to(dev)     # [C, n + 4]
        nk = host[:, n + 1].to(torch.int32)
        cols = torch.gather(host[:, :n], 1, sig)
        cols.masked_fill_(torch.arange(n, device=dev)[None, :] >= nk[:, None], 0)
        out_row = host[:, n].contiguous()
    if bool(one.any()):
        # streams of the one-photon groups, group by group in sorted order, ascending within a group
        idx = torch.nonzero(one)[:, 0]
        idx = idx[torch.sort(inv[idx], stable=True).indices]
        photon = torch.nonzero(kept[inv[idx]])[:, 1]
        s_ids = idx.to(dev)
        s_rows = route_lone_photons(U, dp_all[s_ids].cpu(), im_of(in_modes)[photon], generator=gen).to(dev)
    if not C:
        z = torch.zeros(0, dtype=torch.int64, device=dev)
        return ChainPlan(S, n, 0, z, z.reshape(0, n), z.to(torch.int32), z.reshape(0, n), z, z, z, z, s_ids, s_rows, [])
    order = torch.argsort(nk.to(torch.int64), descending=True, stable=True)
    return ChainPlan(S, n, C, dp_all[out_row], cols, nk, seeds, host[:, n + 2].contiguous(),
                     host[:, n + 3].contiguous(), out_row, order, s_ids, s_rows, passes)


def im_of(in_modes) -> torch.Tensor:
    return torch.as_tensor([int(j) for j in in_modes], dtype=torch.int64)


def assemble_occupations(plan: ChainPlan, rows, m: int) -> torch.Tensor:
    """Occupations [S, m] from the chains' ordered rows [C, n] (first nk entries valid) and the singletons."""
    dev = plan.dp.device
    occ = torch.zeros(plan.S, m, dtype=torch.int64, device=dev)
    if plan.single_ids is not None:
        occ.index_put_((plan.single_ids, plan.single_rows), torch.ones_like(plan.single_rows), accumulate=True)
    if plan.C > 0:
        rows = torch.as_tensor(rows, dtype=torch.int64, device=dev)
        nk = plan.nk if plan.nk is not None else torch.full((plan.C,), plan.n, dtype=torch.int32, device=dev)
        valid = torch.arange(plan.n, device=dev)[None, :] < nk[:, None]
        out = plan.out_row if plan.out_row is not None else torch.arange(plan.C, device=dev)
        occ.index_put_((out[:, None].expand(-1, plan.n)[valid], rows[valid]), torch.ones_like(rows[valid]),
                       accumulate=True)
    return occ
