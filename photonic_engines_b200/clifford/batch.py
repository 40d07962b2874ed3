"""Batched sampler: many independent circuits (different m and n), lossy and partially distinguishable
shots, in ONE persistent chain launch, replayed as a captured CUDA graph.

    bs = BatchedSampler([(U_0, modes_0), (U_1, modes_1), ...], shots=1000, loss=[0.8, 0.9, ...],
                        indist=None, precision="mixed", seed=0)
    occ = bs.sample()                  # [S_total, m_max] int64; rows of circuit g are bs.rows_of(g)

One replay is: fresh Philox key and per-step seeds from the device generator, the device-side partition
of every shot into chains (`pe_partition_shots`: lost photons dropped, interfering photons in a uniform
random order, lone photons as one-photon chains), longest chains first, the chain kernel over all chains,
and the occupations (`pe_scatter_occupations`).  No host work and no host synchronisation per batch.
The law is the reference's (lossy / x-model partially distinguishable Fock sampling); the draws are not
the reference's host draws — `fock_sample` is the path that reproduces those.  The reference's
equivalent is one `fock_sample(..., loss=eta_g)` call per circuit.
"""
from __future__ import annotations

import math

import torch

from .. import _native as N
from .. import autotune
from .kernels import (WARP_MAX_PHOTONS, _split_slots, default_tpl, effective_precision, pack_ragged, split_plan,
                      use_warp_form)


def _resident_split_ctas(device, precision: str, n: int, tpl: int) -> int:
    dev = torch.device(device)
    return _split_slots(dev.index if dev.index is not None else torch.cuda.current_device(), precision, n, 128, tpl)

DEFAULT_CUTS = (20, 16)
WARP_SMALL = 8                 # warp-form batches: chains of at most this many photons get their own tier
LONG_SPLIT_ABOVE = 24          # chains longer than this get their own tier with split steps
# tier cut points the autotuner tries (descending; the last tier <= 16 photons runs in the warp form)
CUT_CANDIDATES = [(20, 16), (24, 16), (20, 12), (24, 20, 16), (16,), (20, 16, 12)]


def _per_instance(v, G, default):
    if v is None:
        return [default] * G
    if isinstance(v, (list, tuple)):
        if len(v) != G:
            raise ValueError(f"one value per circuit ({G}) expected, got {len(v)}")
        return [default if x is None else float(x) for x in v]
    return [float(v)] * G


class BatchedSampler:
    """Exact samples of G independent circuits in one launch per batch (see the module docstring).

    circuits: [(U_g [m_g, m_g] complex CUDA tensor, in_modes_g)], shots: int or per-circuit list,
    loss: transmission eta (scalar or per circuit), indist: x-model overlap x (scalar or per circuit),
    precision: "f64" | "mixed" | "compensated", seed: seeds the device generator, graph: capture the batch in a CUDA graph,
    tune: pick the launch shape with the autotuner (cached per GPU and workload); tiers: run chains of
    different lengths in kernels sized to them (False: one launch sized to the longest).
    """

    def __init__(self, circuits, shots, loss=None, indist=None, precision: str = "mixed", seed: int = 0,
                 graph: bool = True, tune: bool = True, block_threads: int = 0, tpl: int = 0, tiers: bool = True):
        if not circuits:
            raise ValueError("at least one circuit")
        if precision not in N.PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}: 'f64', 'mixed' or 'compensated'")
        U0 = circuits[0][0]
        N.require_cuda(U0, "U")
        self.device = U0.device
        dev = self.device
        G = len(circuits)
        for U, modes in circuits:
            if U.dim() != 2 or U.shape[0] != U.shape[1]:
                raise ValueError("every U must be a square [m, m] matrix")
            if any(not 0 <= int(j) < U.shape[0] for j in modes):
                raise ValueError("input modes must be modes of their circuit")
        shots_l = [int(shots)] * G if not isinstance(shots, (list, tuple)) else [int(x) for x in shots]
        if len(shots_l) != G or any(x < 0 for x in shots_l):
            raise ValueError("shots: one non-negative count per circuit")
        etas = _per_instance(loss, G, 1.0)
        xs = _per_instance(indist, G, 1.0)
        if any(not 0.0 <= e <= 1.0 for e in etas) or any(not 0.0 <= x <= 1.0 for x in xs):
            raise ValueError("loss (transmission) and indist (x-model overlap) must lie in [0, 1]")
        self.G = G
        self.shots = shots_l
        self.m = [int(U.shape[0]) for U, _ in circuits]
        self.n = [len(modes) for _, modes in circuits]
        self.m_max, self.n_stride = max(self.m), max(max(self.n), 1)
        N.check_photons(self.n_stride, precision, "photons per circuit")
        self.precision = precision = effective_precision(precision, self.n_stride)
        self.S = sum(shots_l)
        self.acol, self.inst_off, self.inst_m, self.inst_n = pack_ragged(circuits)
        self.acol = torch.view_as_real(self.acol).contiguous()
        self.dp = torch.repeat_interleave(torch.arange(G, device=dev), torch.tensor(shots_l, device=dev)).contiguous()
        self.eta = torch.tensor(etas, dtype=torch.float64, device=dev)
        self.x = torch.tensor(xs, dtype=torch.float64, device=dev)
        self.singles = any(x < 1.0 for x in xs)
        slots = 1 + self.n_stride if self.singles else 1
        self.C = self.S * slots
        S, C, ns = self.S, self.C, self.n_stride
        self.key = torch.zeros(1, dtype=torch.int64, device=dev)
        self.seeds = torch.zeros(1, ns, dtype=torch.int64, device=dev)
        self.cols = torch.zeros(C, ns, dtype=torch.int64, device=dev)
        self.nk = torch.zeros(C, dtype=torch.int32, device=dev)
        self.chain_dp = torch.zeros(C, dtype=torch.int64, device=dev)
        self.out_row = torch.zeros(C, dtype=torch.int64, device=dev)
        self.order = torch.arange(C, dtype=torch.int64, device=dev)
        self.nk_sorted = torch.zeros(C, dtype=torch.int32, device=dev)
        self.rows = torch.zeros(C, ns, dtype=torch.int64, device=dev)
        self.occ = torch.zeros(S, self.m_max, dtype=torch.int64, device=dev)
        self.status = torch.zeros(2, dtype=torch.int32, device=dev)
        # short chains: one warp per stream (FP64 and mixed forms; the compensated form runs CTAs only)
        self.warp = precision != "compensated" and use_warp_form(self.S, self.n_stride, dev)
        self.split = None if self.warp else split_plan(self.S, self.n_stride, dev, 0,           # few long chains
                                                        default_tpl(self.n_stride, precision), precision)
        if self.split:
            self.ws = torch.empty(int(N.load().pe_chain_split_workspace_bytes(C, self.split[1])), dtype=torch.uint8,
                                  device=dev)
        else:
            self.ws = N.workspace(dev)
        # length tiers: when the chains of a batch differ in length (loss, singles, circuits of several n),
        # every chain runs in the smallest kernel that holds it — the length-sorted order is cut on the device
        # at the tier cut points (default > 20, 17..20 and <= 16 photons, the last in the warp form), one
        # launch per tier on its own stream with its own workspace (pe_fock_chain_range), so the graph
        # replays the cut for every batch; the autotuner may pick other cut points
        varied = self.singles or any(e < 1.0 for e in etas) or len(set(self.n)) > 1
        self.tiered = bool(tiers and varied and not self.warp and not self.split and self.n_stride > WARP_MAX_PHOTONS)
        # short chains of several lengths, all in the warp form: those of at most 8 photons in the 8-column
        # kernel (smaller shared-memory slices, three CTAs per SM), the rest in the batch's own
        self.warp_tiered = bool(tiers and varied and self.warp and self.n_stride > WARP_SMALL)
        self.wsb = int(N.load().pe_chain_workspace_bytes(C))
        self.qr_all = torch.tensor([0, C], dtype=torch.int64, device=dev)      # the whole queue (warp form)
        self.tier_ws, self._side_streams = [], []
        self.long_split = self._plan_long_split(etas, xs) if self.tiered else None
        self._set_tiers(DEFAULT_CUTS if self.tiered else ((WARP_SMALL,) if self.warp_tiered else ()))
        self.gen = torch.Generator(device=dev).manual_seed(seed)
        self._row0 = [0]
        for s_ in shots_l:
            self._row0.append(self._row0[-1] + s_)
        self.tpl, self.block = tpl, block_threads
        self.warp_block = 0                                          # streams per CTA of a warp-form tier x 32
        self.graph = None
        if tune and self.tiered:
            self._tune_cuts()
        if tune and not (tpl and block_threads):
            self._autotune()
        self.graph = None
        if graph:
            self._capture()

    def _set_tiers(self, cuts):
        """Tiers for cut points `cuts` (descending photon counts): chains above cuts[0] in the batch's own
        kernel, then one tier per interval, the last (<= cuts[-1], at most 16 photons) in the warp form for
        the FP64 and mixed forms.  Empty `cuts`: no tiers."""
        dev = self.device
        cuts = tuple(c for c in cuts if c < self.n_stride)
        self.cuts = cuts
        self.tiers = []
        if not cuts:
            return
        last_warp = 1 if (cuts[-1] <= WARP_MAX_PHOTONS and self.precision != "compensated") else 0
        top = 1 if self.warp else 0                      # a warp-form batch keeps its longest chains in it too
        self.tiers = [(self.n_stride, top)] + [(c, 0) for c in cuts[:-1]] + [(cuts[-1], last_warp)]
        if self.long_split is not None:                  # the longest chains: their own tier, steps split
            lim = self.long_split["above"]
            self.tiers = [(self.n_stride, 2)] + [t for t in self.tiers if t[0] < lim]
            if self.tiers[1][0] != lim:
                self.tiers.insert(1, (lim, 0))
        self.tier_thr = torch.tensor([t[0] for t in self.tiers[1:]], dtype=torch.int32, device=dev)
        self.qr = torch.zeros(len(self.tiers), 2, dtype=torch.int64, device=dev)
        self.qr[-1, 1] = self.C                                      # the cuts between tiers move per batch
        # workspaces and side streams are made once, as many as the most tiers any cut set gives, and reused
        if self.long_split is not None and not self.tier_ws:
            self.tier_ws.append(torch.zeros(self.long_split["ws_bytes"], dtype=torch.uint8, device=dev))
        while len(self.tier_ws) < len(self.tiers):
            self.tier_ws.append(torch.zeros(self.wsb, dtype=torch.uint8, device=dev))
        while len(self._side_streams) < len(self.tiers) - 1:
            self._side_streams.append(torch.cuda.Stream(dev))
        self.tier_streams = self._side_streams[:len(self.tiers) - 1]

    def _plan_long_split(self, etas, xs):
        """The split tier of the longest chains (more than LONG_SPLIT_ABOVE photons), or None: expected count E
        of such chains per batch (every photon of circuit g interferes with probability eta_g x_g), slots
        4 E + 64 (positions past them run whole in the persistent kernel), nch a power of two with E nch at
        least four times the split kernel's resident CTAs, k_split the first step with 4 nch lanes' worth of
        Gray terms.  A chain of 27 photons holds one CTA for about 0.3 s, as long as all other chains of a
        100 000-shot batch together; split, its heavy steps run on nch CTAs."""
        above = LONG_SPLIT_ABOVE
        if self.n_stride <= above:
            return None
        E = 0.0
        for n_g, sh, e_, x_ in zip(self.n, self.shots, etas, xs):
            q = e_ * x_
            E += sh * sum(math.comb(n_g, j) * q ** j * (1.0 - q) ** (n_g - j) for j in range(above + 1, n_g + 1))
        slots = int(min(self.C, 4 * E + 64))
        tpl = default_tpl(self.n_stride, self.precision)
        resident = _resident_split_ctas(self.device, self.precision, self.n_stride, tpl)
        nch = 4
        while nch < 128 and max(E, 1.0) * nch < 4 * resident:
            nch *= 2
        lanes = 128 // tpl
        k = 2
        while k <= self.n_stride and (1 << (k - 2)) < 4 * nch * lanes:
            k += 1
        if k > self.n_stride:
            return None
        wsb = int(N.load().pe_range_split_workspace_bytes(slots, nch))
        return {"above": above, "slots": slots, "nch": nch, "k_split": k, "expected": E, "ws_bytes": wsb}

    # ---------------------------------------------------------------------------------------- one batch
    def _draw_keys(self):
        r = torch.randint(0, 2 ** 31 - 1, (1 + self.n_stride,), generator=self.gen, device=self.device)
        self.key.copy_(r[:1])
        self.seeds.copy_(r[1:].view(1, -1))

    def _partition(self):
        st = N.stream_handle(self.device)
        L = N.load()
        N.check(L.pe_partition_shots(N.ptr(self.dp), N.ptr(self.inst_n), N.ptr(self.eta), N.ptr(self.x), self.S,
                                     self.n_stride, int(self.singles), N.ptr(self.key), N.ptr(self.cols), N.ptr(self.nk),
                                     N.ptr(self.chain_dp), N.ptr(self.out_row), N.ptr(self.status[:1]), st),
                "pe_partition_shots")
        torch.sort(self.nk, descending=True, stable=True, out=(self.nk_sorted, self.order))   # longest chains first

    def _chains(self, tpl=None, block=None):
        st = N.stream_handle(self.device)
        L = N.load()
        common = (N.PRECISIONS[self.precision], N.ptr(self.acol), N.ptr(self.inst_off), N.ptr(self.inst_m),
                  N.ptr(self.inst_n), self.G, self.m_max, self.C, N.ptr(self.chain_dp), N.ptr(self.nk), N.ptr(self.cols),
                  self.n_stride, None, N.ptr(self.seeds), None, None, N.ptr(self.order), N.ptr(self.rows), None,
                  self.m_max, None, self.m_max)
        block = int(self.block if block is None else block)
        tpl = int(self.tpl if tpl is None else tpl)
        if self.tiers:
            cnt = (self.nk_sorted.unsqueeze(0) > self.tier_thr.unsqueeze(1)).sum(1)    # chains above each cut
            self.qr[1:, 0] = cnt
            self.qr[:-1, 1] = cnt
            cur = torch.cuda.current_stream(self.device)
            for s_ in self.tier_streams:
                s_.wait_stream(cur)
            for i, (nk_max, mode) in enumerate(self.tiers):
                stream = cur if i == 0 else self.tier_streams[i - 1]
                b, t = (block, tpl) if i == 0 else (0, 0)          # the tuned shape is the top tier's
                if mode == 1 and i == 0:                          # a warp-form batch's longest chains
                    t = tpl if tpl in (1, 2) else 0
                elif mode == 1:
                    b, t = self.warp_block, 0
                if mode == 2:
                    ls = self.long_split
                    rc = L.pe_fock_chain_range_split(*common, N.ptr(self.tier_ws[i]), self.tier_ws[i].numel(), b, t,
                                                     N.ptr(self.qr[i]), nk_max, ls["k_split"], ls["nch"],
                                                     ls["slots"], stream.cuda_stream)
                    N.check(rc, "pe_fock_chain_range_split")
                    continue
                rc = L.pe_fock_chain_range(*common, N.ptr(self.tier_ws[i]), self.tier_ws[i].numel(), b, t, 0,
                                           N.ptr(self.qr[i]), nk_max, mode, stream.cuda_stream)
                N.check(rc, "pe_fock_chain_range")
            for s_ in self.tier_streams:
                cur.wait_stream(s_)
            return
        if self.warp:                  # the whole queue in the warp form, block / 32 streams per CTA
            rc = L.pe_fock_chain_range(*common, N.ptr(self.ws), self.ws.numel(), block, tpl if tpl in (1, 2) else 0,
                                       0, N.ptr(self.qr_all), self.n_stride, 1, st)
        elif self.split:
            rc = L.pe_fock_chain_split(*common, self.split[0], self.split[1], N.ptr(self.ws), self.ws.numel(), block,
                                       tpl, st)
        else:
            rc = L.pe_fock_chain(*common, N.ptr(self.ws), self.ws.numel(), block, tpl, 0, st)
        N.check(rc, "pe_fock_chain")

    def _scatter(self):
        N.check(N.load().pe_scatter_occupations(N.ptr(self.rows), N.ptr(self.nk), N.ptr(self.out_row), self.C,
                                                self.n_stride, N.ptr(self.occ), self.m_max, self.S,
                                                N.ptr(self.status[1:]), N.stream_handle(self.device)),
                "pe_scatter_occupations")

    def _step(self):
        self._draw_keys()
        self._partition()
        self._chains()
        self._scatter()

    def _tune_cuts(self):
        """Pick the tier cut points: every candidate set is captured as the batch's CUDA graph and timed by
        whole-batch replays (the tiers run concurrently on their streams, so only the replayed graph times
        them as they run), the fastest kept — the default unless another set is more than 3 % faster — and
        cached per GPU and workload like the launch shape."""
        workload = (f"cuts|G{self.G}|S{self.S}|m{self.m_max}|n{self.n_stride}|singles{int(self.singles)}|"
                    f"{self.precision}")
        cands = [c for c in CUT_CANDIDATES if all(x < self.n_stride for x in c)] or [DEFAULT_CUTS]

        def run(i, _block):
            if self.graph is None or self.cuts != tuple(c for c in cands[i] if c < self.n_stride):
                self._set_tiers(cands[i])                  # switched (and captured) in the warm-up call
                self._capture()
            self.graph.replay()
        best = autotune.tune(run, self.device, self.precision, 0, workload,
                             candidates=[(i, 0) for i in range(len(cands))], reps=3, keep_first_within=0.03)
        self.graph = None
        self._set_tiers(cands[best[0]])

    def _autotune(self):
        workload = (f"batch|G{self.G}|S{self.S}|m{self.m_max}|n{self.n_stride}|singles{int(self.singles)}|"
                    f"{'warp' if self.warp else 'cta'}|tiers{len(self.tiers)}")
        self._draw_keys()
        self._partition()
        if self.warp:
            best = autotune.tune(lambda tpl, block: self._chains(tpl, block), self.device, self.precision,
                                 autotune.tier(self.n_stride), workload, candidates=autotune.WARP_CANDIDATES)
        else:
            best = autotune.tune(lambda tpl, block: self._chains(tpl, block), self.device, self.precision,
                                 autotune.tier(self.n_stride), workload + f"|cuts{self.cuts}")
            if self.tiers and self.tiers[-1][1]:                     # streams per CTA of the warp-form tier
                def run_warp(_tpl, block):
                    self.warp_block = block
                    self._chains()
                wb = autotune.tune(run_warp, self.device, self.precision, 16, workload + f"|cuts{self.cuts}|warptier",
                                   candidates=[(0, b) for b in (64, 128, 256)])
                self.warp_block = wb[1]
        self.tpl, self.block = best

    def _capture(self):
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            for _ in range(2):
                self._step()
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        g.register_generator_state(self.gen)
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            self._step()
        self.graph = g

    # ---------------------------------------------------------------------------------------- public
    def sample(self) -> torch.Tensor:
        """Run one batch; returns the occupations [S_total, m_max] (a buffer reused by the next call)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._step()
        return self.occ

    def rows_of(self, g: int) -> slice:
        """Rows of circuit g in the occupation buffer (its modes are columns 0..m_g - 1)."""
        return slice(self._row0[g], self._row0[g + 1])

    def check(self) -> None:
        """Raise when a device-side index error was recorded (synchronises)."""
        st = self.status.cpu().tolist()
        ws = 0
        for w in (self.tier_ws[:len(self.tiers)] if self.tiers else [self.ws]):
            ws = ws or N.read_status(w)[0]
        if any(st) or ws:
            raise N.NativeError(f"device-side error in the batched sampler (partition {st[0]}, scatter {st[1]}, "
                                f"chains {ws})")
