#!/usr/bin/env python
"""Benchmark of the exact Fock sampler on B200: samples/s at n = 20, m = 400 (2 000 shots per step,
lossless, Haar-random U) in three forms — FP64, mixed (plain FP32 Gray blocks) and compensated mixed
(double-float FP32 Gray blocks) — with each FP32 form's marginal error against the FP64 form on the same
chains.  `value` is the fastest form whose maximum marginal relative error is within the metric's bound
(1e-6); every form's figures are under `forms`, and `configs` carries the c3 / c4 / c5 configurations
run through the batched sampler.

    python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference]

A step is one pass of the sampling path over one batch: sigma and per-step seeds drawn from the device
generator, then the whole chains of all 2 000 shots in one launch of the persistent chain kernel.
`value` times K steps with inputs resident in HBM (L2 flushed between steps by a 256 MiB write);
`e2e` times the public `fock_sample` call with U copied from pinned host memory and the occupations
copied back every step.  Under torchrun every rank runs its own replica (weak scaling, no collective
on the data path); the time is the max over ranks.  `--impl reference` times the CPU restatement of the
reference's algorithm (oracle/, all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_PHOT, M_MODES, SHOTS, USEED = 20, 400, 2000, 1002
# DRAM bytes (read + write) of one chain launch on this workload, from one ncu capture of each form
# (dram__bytes_read.sum + dram__bytes_write.sum, `--profile-launch f64|mixed|compensated`); the algorithmic bytes
# (16 m k + 16 k^2 per sample and step, 2.78 GB per launch) are served from L2 and shared memory.
DRAM_BYTES_PER_LAUNCH = {"f64": 1.119e6 + 0.0, "mixed": 1.008e6 + 0.023e6, "compensated": 0.807e6 + 0.0}
METRIC = "samples/s n=20 m=400: mixed-precision vs FP64 on B200, marginal err<=1e-6"
BOUND = 1e-6                                    # the metric's marginal error bound
FORMS = ("f64", "mixed", "compensated")         # FP64 first: the reference every other form is measured against
DTYPES = {"f64": "f64", "mixed": "f32 Gray blocks + f64 sums/marginal/CDF",
          "compensated": "f32 double-float Gray blocks + f64 sums/marginal/CDF"}
SMS_B200 = 148
NOMINAL_LANES = {"f64": 64, "mixed": 128}      # FMA lanes per SM per clock
WORKLOAD = "fock n=20 photons (modes 0..19), m=400, 2000 shots/step, lossless, Haar U (seeded QR)"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ----------------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        except (OSError, ValueError):
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------------------- reference arm
def run_reference(args):
    """The CPU restatement of the reference's algorithm (oracle/, C, all host threads) on a bounded sample:
    every step samples `--ref-shots` chains of the benchmark workload."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    import numpy as np

    from oracle import oracle as O
    U = O.haar_unitary(M_MODES, USEED)
    A = U[:, :N_PHOT]
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(0)
    # the benchmark's own 2 000 chains per step when the whole run stays near 150 s on this port (about 17
    # chains/s per host thread at n = 20, m = 400), else fewer per step
    S = args.ref_shots or max(64, min(SHOTS, int(150 * 17 * threads / max(1, args.steps + args.warmup))))

    def step():
        sig = np.argsort(rng.random((S, N_PHOT)), axis=1)
        u = rng.random((S, N_PHOT))
        O.chain(A, np.zeros(S, np.int64), sig, u, threads=threads)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = args.steps * S / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": N_PHOT, "m": M_MODES, "shots_per_step": S, "precision": "f64"},
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": threads, "kind": "port",
                             "sample": f"{S} chains per step of the n=20 m=400 workload (bounded sample)"},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_torch_sampler": reference_torch_sampler(),
            "reference_gpu": None if args.no_reference_gpu else reference_engine_gpu()}
    print(json.dumps(line), flush=True)


def reference_engine_gpu() -> dict:
    """The reference's own GPU engine (its public fock_sample, default Triton backend, unmodified, from
    baseline/_ref) on this machine's GPU at the benchmark workload: 2 000 shots per call, 3 timed calls.
    Only the reference's code runs here."""
    import torch
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    U = _haar_dev(M_MODES, USEED, torch.device("cuda"))
    return public_call_leg([(U, list(range(N_PHOT)))], SHOTS, reps=3, ours=False)


def _reference_fock_sample():
    """The reference's public fock_sample from its offline install in baseline/_ref, or (None, why)."""
    ref = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref, "photonic_engines")):
        return None, "baseline/_ref holds no install of the reference"
    try:
        import triton  # noqa: F401
    except ImportError:
        return None, "triton is not importable (the reference's GPU engine is Triton)"
    sys.path.insert(0, ref)
    try:
        import photonic_engines.clifford as rc
    finally:
        sys.path.remove(ref)
    return rc.fock_sample, None


def public_call_leg(circuits, shots, loss=None, indist=None, reps: int = 1, ours: bool = True,
                    extra: dict | None = None) -> dict:
    """One public sampling call per circuit, through the reference's own GPU engine (its fock_sample with its
    default Triton backend, unmodified, from baseline/_ref) and, with `ours`, through this library's
    fock_sample (FP64, the drop-in), from equal CUDA generator seeds on this GPU.  Per engine: samples/s over
    `reps` timed rounds (CUDA events, after one untimed round that also builds the reference's Triton
    kernels); and how many occupation rows of the last round agree between the two."""
    import torch
    ref_fn, why = _reference_fock_sample()
    if ref_fn is None:
        return {"unavailable": why}
    engines = [("reference", ref_fn)]
    if ours:
        from photonic_engines_b200.clifford import fock_sample
        engines.append(("fock_sample", fock_sample))
    total = shots * len(circuits)

    def run(fn, seed):
        outs = []
        for i, (U, modes) in enumerate(circuits):
            kw = {}
            if loss is not None:
                kw["loss"] = loss[i] if isinstance(loss, list) else loss
            if indist is not None:
                kw["indist"] = indist
            kw.update(extra or {})
            outs.append(fn(U, modes, shots, generator=torch.Generator(device=U.device).manual_seed(seed + i), **kw))
        return outs

    res, last = {}, {}
    for name, fn in engines:
        run(fn, 1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for r in range(reps):
            last[name] = run(fn, 7 + 100000 * r)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        res[name] = {"value": total / (ms * 1e-3), "unit": "samples/s", "ms_per_call_round": ms}
    res["reference"]["engine"] = "reference photonic_engines.clifford.fock_sample, backend triton (its default)"
    if ours:
        same, rows = 0, 0
        for a, b in zip(last["reference"], last["fock_sample"]):
            if isinstance(a, tuple):                 # keep_ids: (occupations, surviving stream ids)
                if not torch.equal(a[1].cpu(), b[1].cpu()):
                    rows += a[0].shape[0]
                    continue
                a, b = a[0], b[0]
            same += int((a.cpu() == b.cpu()).all(dim=1).sum()) if a.shape == b.shape else 0
            rows += a.shape[0]
        res["identical_rows"] = same
        res["rows"] = rows
    res["calls_per_round"] = len(circuits)
    return res


def reference_torch_sampler(shots: int = 1) -> dict:
    """The reference's own CPU sampler for this path, unmodified, from its offline install in baseline/_ref:
    variants.fock_sample_reference (photonic_engines/clifford/variants.py:218-241, pure torch, FP64) on `shots`
    shots of the benchmark workload (about 13 s per shot on 8 host threads), as samples/s."""
    ref = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref, "photonic_engines")):
        return {"unavailable": "baseline/_ref holds no install of the reference"}
    import torch
    sys.path.insert(0, ref)
    try:
        from photonic_engines.clifford import variants
    finally:
        sys.path.remove(ref)
    g = torch.Generator().manual_seed(USEED)
    z = torch.randn(M_MODES, M_MODES, generator=g, dtype=torch.float64) + 1j * torch.randn(
        M_MODES, M_MODES, generator=g, dtype=torch.float64)
    q, r = torch.linalg.qr(z)
    d = torch.diagonal(r)
    U = q * (d / d.abs()).unsqueeze(0)
    t0 = time.perf_counter()
    occ = variants.fock_sample_reference(U, list(range(N_PHOT)), shots, algo="2020",
                                         generator=torch.Generator().manual_seed(3))
    dt = time.perf_counter() - t0
    assert int(occ.sum()) == shots * N_PHOT
    return {"value": shots / dt, "unit": "samples/s", "cores": torch.get_num_threads(), "kind": "reference",
            "sample": f"{shots} shot(s) of the n=20 m=400 workload through the reference's variants."
                      f"fock_sample_reference (torch CPU, FP64), {dt:.1f} s"}


# ----------------------------------------------------------------------------------------- B200 arm
def run_b200(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from photonic_engines_b200 import _native as NAT
    from photonic_engines_b200 import replicas as REP
    from photonic_engines_b200.clifford import fock_sample
    from photonic_engines_b200.clifford.kernels import chain, pack_instances
    from photonic_engines_b200.clifford.work import chain_work

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    REP.init("nccl", device=dev)
    g = torch.Generator().manual_seed(USEED)
    z = torch.randn(M_MODES, M_MODES, generator=g, dtype=torch.float64) + 1j * torch.randn(
        M_MODES, M_MODES, generator=g, dtype=torch.float64)
    q, r = torch.linalg.qr(z)
    d = torch.diagonal(r)
    U_host = (q * (d / d.abs()).unsqueeze(0)).contiguous()
    U = U_host.to(dev)
    in_modes = list(range(N_PHOT))
    acol, off, mm, nn = pack_instances(U, in_modes)
    dp = torch.zeros(SHOTS, dtype=torch.int64, device=dev)
    gen = torch.Generator(device=dev).manual_seed(REP.replica_seed(1000, rank))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    rows_buf = torch.empty(SHOTS, N_PHOT, dtype=torch.int64, device=dev)
    occ_buf = torch.empty(SHOTS, M_MODES, dtype=torch.int64, device=dev)

    def step(precision, marg=None):
        sig = torch.argsort(torch.rand(SHOTS, N_PHOT, generator=gen, device=dev), dim=1)
        seeds = torch.randint(0, 2 ** 31 - 1, (N_PHOT,), generator=gen, device=dev)
        rows, _, mg = chain(acol, off, mm, nn, dp, sig, m_max=M_MODES, seeds=seeds, precision=precision,
                            want_marg=marg is not None, check_status=False,
                            out=(rows_buf, occ_buf, marg) if marg is not None else (rows_buf, occ_buf, None))
        return sig, seeds, rows

    def barrier():
        if ws > 1:
            dist.barrier()

    max_over_ranks = REP.max_over_ranks

    def timed(precision, steps, warmup):
        for _ in range(warmup):
            step(precision)
        torch.cuda.synchronize(dev)
        kern_ms, work, all_rows = [], [], []
        barrier()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        evs = []
        with ClockSampler(local) as clk:
            e0.record()
            for _ in range(steps):
                flush.fill_(1)
                sig = torch.argsort(torch.rand(SHOTS, N_PHOT, generator=gen, device=dev), dim=1)
                seeds = torch.randint(0, 2 ** 31 - 1, (N_PHOT,), generator=gen, device=dev)
                k0 = torch.cuda.Event(enable_timing=True)
                k1 = torch.cuda.Event(enable_timing=True)
                k0.record()
                rows, _, _ = chain(acol, off, mm, nn, dp, sig, m_max=M_MODES, seeds=seeds, precision=precision,
                                   want_occ=True, check_status=False)
                k1.record()
                evs.append((k0, k1))
                all_rows.append(rows)
            e1.record()
            torch.cuda.synchronize(dev)
        barrier()
        elapsed = e0.elapsed_time(e1) * 1e-3
        kern_ms = [a.elapsed_time(b) for a, b in evs]
        wk = [chain_work(r.cpu().numpy(), M_MODES) for r in all_rows]
        return {"elapsed": max_over_ranks(elapsed), "kern_ms": kern_ms, "work": wk, "clocks": clk.summary()}

    peak = {"f64": NAT.pipe_peak_tflops("f64", dev), "mixed": NAT.pipe_peak_tflops("mixed", dev)}
    peak["compensated"] = peak["mixed"]
    res = {}
    for precision in FORMS:
        res[precision] = timed(precision, args.steps, args.warmup)

    # marginal error of each FP32 form against the FP64 form on the same chains (same sigma, same seeds);
    # the FP64 form itself is held within 1e-10 of the long-double oracle by the parity tests
    sig = torch.argsort(torch.rand(256, N_PHOT, generator=gen, device=dev), dim=1)
    seeds = torch.randint(0, 2 ** 31 - 1, (N_PHOT,), generator=gen, device=dev)
    dp256 = torch.zeros(256, dtype=torch.int64, device=dev)
    r64, _, m64 = chain(acol, off, mm, nn, dp256, sig, m_max=M_MODES, seeds=seeds, precision="f64", want_marg=True)
    err, picks_equal, err_by_k = {"f64": 0.0}, {"f64": True}, {}
    for precision in FORMS[1:]:
        r, _, mg = chain(acol, off, mm, nn, dp256, sig, m_max=M_MODES, seeds=seeds, precision=precision,
                         want_marg=True)
        e = (mg - m64).abs().amax(dim=2) / m64.abs().amax(dim=2)           # [chains, steps]
        err[precision] = float(e.max())
        err_by_k[precision] = [float(x) for x in e.amax(dim=0)]
        picks_equal[precision] = bool(torch.equal(r64, r))
    value = {f: ws * SHOTS * args.steps / res[f]["elapsed"] for f in FORMS}
    meets = {f: err[f] <= BOUND for f in FORMS}
    head = max((f for f in FORMS if meets[f]), key=lambda f: value[f])

    # end to end through the public API in the headline form: U from pinned host memory, occupations back
    U_pin = U_host.pin_memory()
    out_pin = torch.empty(SHOTS, M_MODES, dtype=torch.int64).pin_memory()
    gen_e2e = torch.Generator(device=dev).manual_seed(REP.replica_seed(7, rank))

    def e2e_step():
        Ud = U_pin.to(dev, non_blocking=True)
        occ = fock_sample(Ud, in_modes, SHOTS, generator=gen_e2e, precision=head)
        out_pin.copy_(occ, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize(dev)
    barrier()
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ee0.record()
    for _ in range(args.steps):
        e2e_step()
    ee1.record()
    torch.cuda.synchronize(dev)
    e2e_elapsed = max_over_ranks(ee0.elapsed_time(ee1) * 1e-3)

    configs = None
    if rank == 0 and ws == 1 and not args.no_configs:
        configs = {name: config_result(name, min(args.steps, 3), 3, not args.no_reference_gpu)
                   for name in ("c3", "c4", "c5")}

    # the same public call through the reference's own GPU engine on this GPU, and row-for-row agreement
    ref_gpu = None
    if rank == 0 and ws == 1 and not args.no_reference_gpu:
        ref_gpu = public_call_leg([(U, in_modes)], SHOTS, reps=3)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.ref_shots or 96 * (os.cpu_count() or 1))

    if rank == 0:
        sm_mhz = res[head]["clocks"].get("sm_max_mhz") or 1965.0
        nominal = {"f64": NOMINAL_LANES["f64"] * 2 * SMS_B200 * sm_mhz * 1e6 / 1e12,
                   "mixed": NOMINAL_LANES["mixed"] * 2 * SMS_B200 * sm_mhz * 1e6 / 1e12}
        nominal["compensated"] = nominal["mixed"]

        def roof(r, form):
            flops_launch = statistics.mean(w["flops"] for w in r["work"])
            dur = statistics.mean(r["kern_ms"]) * 1e-3
            achieved = flops_launch / dur / 1e12
            return {"bound": "fp64" if form == "f64" else "fp32", "achieved": achieved, "peak": peak[form],
                    "unit": "TFLOP/s", "frac": achieved / peak[form],
                    "frac_of_nominal": achieved / nominal[form], "peak_nominal": nominal[form],
                    "traffic": DRAM_BYTES_PER_LAUNCH.get(form),
                    "traffic_unit": "bytes per launch (ncu dram read + write, one capture)",
                    "algorithmic_bytes_per_launch": statistics.mean(w["bytes"] for w in r["work"]),
                    "peak_source": "measured live by pe_pipe_probe (FMA chains) on this GPU; nominal = lanes x 2 "
                                   "x 148 SMs x SM clock",
                    "flops_per_launch": flops_launch, "launch_ms": dur * 1e3}

        forms = {f: {"value": value[f], "ms_per_step": res[f]["elapsed"] / args.steps * 1e3,
                     "roofline": roof(res[f], f), "max_marginal_rel_err": err[f], "meets_bound": meets[f],
                     "picks_equal_fp64": picks_equal[f], "marginal_err_by_k": err_by_k.get(f),
                     "clocks": res[f]["clocks"]} for f in FORMS}
        line = {
            "metric": METRIC, "value": value[head], "unit": "samples/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res[head]["elapsed"] / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPES[head], "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": N_PHOT, "m": M_MODES, "shots_per_step": SHOTS,
                       "precision": head, "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"replicas x{ws}"},
            "headline_form": head, "bound": BOUND,
            "headline_rule": "value = the fastest form whose max marginal relative error (vs the FP64 form, "
                             "256 chains x 20 steps) is <= bound",
            "roofline": roof(res[head], head),
            "forms": forms,
            "fp64": {"value": value["f64"], "ms_per_step": forms["f64"]["ms_per_step"],
                     "roofline": forms["f64"]["roofline"], "clocks": res["f64"]["clocks"]},
            "mixed_over_fp64": value["mixed"] / value["f64"],
            "compensated_over_fp64": value["compensated"] / value["f64"],
            "max_marginal_rel_err": err[head],
            "addends_per_sample": statistics.mean(w["addends"] for w in res[head]["work"]) / SHOTS,
            "cpu_baseline": cpu,
            "e2e": {"value": ws * SHOTS * args.steps / e2e_elapsed, "unit": "samples/s", "precision": head,
                    "h2d_bytes_per_step": U_host.numel() * 16, "d2h_bytes_per_step": SHOTS * M_MODES * 8},
            "clocks": res[head]["clocks"],
            "gpu_launches": args.steps,
            "configs": configs,
            "reference_gpu": ref_gpu,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


def cpu_baseline(S: int) -> dict:
    """The oracle (C restatement of the reference algorithm) on the host cores, bounded sample."""
    import numpy as np

    from oracle import oracle as O
    U = O.haar_unitary(M_MODES, USEED)
    rng = np.random.default_rng(1)
    threads = os.cpu_count() or 1
    sig = np.argsort(rng.random((S, N_PHOT)), axis=1)
    u = rng.random((S, N_PHOT))
    t0 = time.perf_counter()
    O.chain(U[:, :N_PHOT], np.zeros(S, np.int64), sig, u, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": S / dt, "unit": "samples/s", "cores": threads, "kind": "port",
            "sample": f"{S} chains of the n=20 m=400 workload, oracle/ C port, {threads} threads, {dt:.1f} s"}


# ----------------------------------------------------------------------------------------- other configs
def _haar_dev(m: int, seed: int, dev):
    import torch
    g = torch.Generator().manual_seed(seed)
    z = torch.randn(m, m, generator=g, dtype=torch.float64) + 1j * torch.randn(m, m, generator=g, dtype=torch.float64)
    q, r = torch.linalg.qr(z)
    d = torch.diagonal(r)
    return (q * (d / d.abs()).unsqueeze(0)).to(dev)


def _config_circuits(name: str, dev):
    """(circuits, shots, loss, indist, description) of the configurations beside the headline one."""
    import numpy as np
    if name == "c1":
        return [(_haar_dev(12, 1001, dev), list(range(6)))], 10000, None, None, \
            "n=6 m=12, 10000 shots, lossless, Haar U"
    if name == "c3":
        return [(_haar_dev(900, 3001, dev), list(range(30)))], 100000, 0.5, None, \
            "n_in=30 m=900, eta=0.5 (detected k ~ Bin(30, 0.5)), 100000 shots, Haar U"
    if name == "c4":
        return [(_haar_dev(784, 4001, dev), list(range(28)))], 200, None, 0.95, \
            "n=28 m=784, 200 shots, lossless, x-model indist 0.95, Haar U"
    if name == "c5":
        rng = np.random.default_rng(5000)
        circuits, etas = [], []
        for i in range(256):
            m = int(rng.choice([16, 24, 32, 48, 64]))
            n = int(rng.integers(4, min(12, m // 4) + 1))
            circuits.append((_haar_dev(m, 5000 + i, dev), list(range(n))))
            etas.append(float(rng.uniform(0.6, 1.0)))
        return circuits, 1000, etas, None, \
            "256 Haar circuits, m in {16,24,32,48,64}, n in 4..min(12,m/4), eta ~ U[0.6,1], 1000 shots each"
    raise ValueError(name)


def hbm_peak() -> tuple[float, str]:
    """HBM bandwidth denominator: the measured copy bandwidth of this pool's B200s when the peaks file is
    present, else the earlier measurement on this pool."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "of measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "of fallback (6.65 TB/s)"


def config_result(name: str, steps: int, warmup: int, reference_gpu: bool = True) -> dict:
    """One configuration run through the batched sampler (one persistent launch per batch, CUDA-graph
    replay) in every form: samples/s, roofline of the chain kernel, end to end with the occupations copied
    to the host, occupations equal to the FP64 form's, and the marginal error of the FP32 forms against
    the FP64 form by step on lossless chains of the configuration's circuits (supplied uniforms)."""
    import numpy as np
    import torch

    from photonic_engines_b200 import _native as NAT
    from photonic_engines_b200.clifford import BatchedSampler, sample_chains
    from photonic_engines_b200.clifford.work import chain_work

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    circuits, shots, loss, indist, desc = _config_circuits(name, dev)
    peak = {"f64": NAT.pipe_peak_tflops("f64", dev), "mixed": NAT.pipe_peak_tflops("mixed", dev)}
    peak["compensated"] = peak["mixed"]
    out, occs = {}, {}
    for precision in FORMS:
        bs = BatchedSampler(circuits, shots, loss=loss, indist=indist, precision=precision, seed=7, tune=True)
        for _ in range(warmup):
            bs.sample()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(0) as clk:
            e0.record()
            for _ in range(steps):
                bs.sample()
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        bs.check()
        nk = bs.nk.cpu().numpy()
        rows = bs.rows.cpu().numpy()
        dpn = bs.chain_dp.cpu().numpy()
        flops = nbytes = 0.0
        for g in range(bs.G):                                # work of the last batch, per circuit (m differs)
            sel = (dpn == g) & (nk > 0)
            if sel.any():
                w = chain_work(rows[sel], bs.m[g], nk[sel])
                flops += w["flops"]
                nbytes += w["bytes"]
        occs[precision] = bs.occ.clone()
        ach = flops / (ms * 1e-3) / 1e12
        hbm, hbm_src = hbm_peak()
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[precision] = {"value": bs.S / (ms * 1e-3), "ms_per_step": ms, "tpl_block": [bs.tpl, bs.block],
                          "tier_cuts": list(bs.cuts), "warp_tier_block": bs.warp_block, "kernels_run": bs.precision,
                          "roofline": {"bound": "fp64" if bs.precision == "f64" else "fp32", "achieved": ach,
                                       "peak": peak[bs.precision], "unit": "TFLOP/s", "frac": ach / peak[bs.precision],
                                       "traffic": None, "peak_source": "measured live by pe_pipe_probe",
                                       "flops_per_launch": flops},
                          "bytes_roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                                             "frac": gbs / hbm, "peak_source": hbm_src,
                                             "bytes_per_launch": nbytes,
                                             "note": "algorithmic bytes of the draws and block gathers (16 m k + "
                                                     "16 k^2 per chain step); the instances are L2-resident"},
                          "clocks": clk.summary()}
        # end to end: the same batch with the occupations copied to pinned host memory every step
        host = torch.empty_like(bs.occ, device="cpu").pin_memory()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            host.copy_(bs.sample(), non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        out[precision]["e2e"] = {"value": bs.S / (e0.elapsed_time(e1) * 1e-3 / steps), "unit": "samples/s",
                                 "h2d_bytes_per_step": 0, "d2h_bytes_per_step": bs.occ.numel() * 8}
        del bs
    # marginal error of the FP32 forms against the FP64 form on lossless chains of each circuit
    rng = np.random.default_rng(3)
    inst = circuits if len(circuits) <= 8 else [circuits[i] for i in range(0, len(circuits), len(circuits) // 16)]
    for precision in FORMS[1:]:
        max_err, per_k = 0.0, {}
        for U, modes in inst:
            n = len(modes)
            S = 8 if n >= 26 else 32
            sig = np.argsort(rng.random((S, n)), axis=1)
            u = rng.random((S, n))
            a = sample_chains(U, modes, sig, uniforms=u, want_marg=True, split=None)
            b = sample_chains(U, modes, sig, uniforms=u, want_marg=True, precision=precision, split=None)
            e = ((b["marg"] - a["marg"]).abs().amax(2) / a["marg"].abs().amax(2)).cpu().numpy()
            max_err = max(max_err, float(e.max()))
            for k in range(n):
                per_k[k + 1] = max(per_k.get(k + 1, 0.0), float(e[:, k].max()))
            out[precision].setdefault("picks_equal_fp64", True)
            out[precision]["picks_equal_fp64"] &= bool(torch.equal(a["rows"], b["rows"]))
        out[precision].update(max_marginal_rel_err=max_err, marginal_err_by_k=per_k, meets_bound=max_err <= BOUND,
                              occupations_equal_fp64=bool(torch.equal(occs[precision], occs["f64"])),
                              over_fp64=out[precision]["value"] / out["f64"]["value"])
    out["f64"].update(max_marginal_rel_err=0.0, meets_bound=True)
    head = max((f for f in FORMS if out[f]["meets_bound"]), key=lambda f: out[f]["value"])
    # the configuration's public calls (one fock_sample per circuit) through the reference's own GPU engine
    # and through this library's drop-in fock_sample, with row-for-row agreement
    ref_gpu = public_call_leg(circuits, shots, loss, indist) if reference_gpu else None
    return {"config": name, "workload": desc, "metric": "samples/s", "unit": "samples/s",
            "value": out[head]["value"], "headline_form": head, "forms": out, "steps": steps, "warmup": warmup,
            "data": "synthetic", "reference_gpu": ref_gpu}


def run_config(args):
    """`--config c1|c3|c4|c5`: one JSON line for that configuration (config_result)."""
    line = config_result(args.config, args.steps, args.warmup, not args.no_reference_gpu)
    line.update(n_gpus=1)
    print(json.dumps(line), flush=True)


def profile_launch(precision: str):
    """One warm-up launch and one launch of the chain kernel on the benchmark workload (for ncu -s 1 -c 1)."""
    import torch

    from photonic_engines_b200.clifford.kernels import chain, pack_instances
    dev = torch.device("cuda")
    g = torch.Generator().manual_seed(USEED)
    z = torch.randn(M_MODES, M_MODES, generator=g, dtype=torch.float64) + 1j * torch.randn(
        M_MODES, M_MODES, generator=g, dtype=torch.float64)
    q, r = torch.linalg.qr(z)
    d = torch.diagonal(r)
    U = (q * (d / d.abs()).unsqueeze(0)).to(dev)
    acol, off, mm, nn = pack_instances(U, list(range(N_PHOT)))
    gen = torch.Generator(device=dev).manual_seed(5)
    for _ in range(2):
        sig = torch.argsort(torch.rand(SHOTS, N_PHOT, generator=gen, device=dev), dim=1)
        seeds = torch.randint(0, 2 ** 31 - 1, (N_PHOT,), generator=gen, device=dev)
        chain(acol, off, mm, nn, torch.zeros(SHOTS, dtype=torch.int64, device=dev), sig, m_max=M_MODES, seeds=seeds,
              precision=precision)
    torch.cuda.synchronize()


def profile_batch(name: str):
    """Three warm-up batches and two timed batches of a configuration through the batched sampler in FP64,
    launched eagerly (no CUDA graph, default launch shapes) so that a profiler sees every tier's launch."""
    import torch

    from photonic_engines_b200.clifford import BatchedSampler
    dev = torch.device("cuda", 0)
    circuits, shots, loss, indist, _ = _config_circuits(name, dev)
    bs = BatchedSampler(circuits, shots, loss=loss, indist=indist, precision="f64", seed=7, tune=False, graph=False)
    for _ in range(3):
        bs.sample()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(2):
        bs.sample()
    e1.record()
    torch.cuda.synchronize()
    bs.check()
    print(json.dumps({"config": name, "ms_per_batch": e0.elapsed_time(e1) / 2, "tiers": bs.tiers,
                      "chains": bs.C}), flush=True)


def run_emitter(args):
    """One JSON line for EmitterMPS inputs: the linear cluster state (caterpillar, spin_gate(pi/2, 0) at every
    emission, emitter traced out) of n = 12 photons in m = 24 modes through a seeded Haar U, 512 shots per step
    — the workload of the reference's bench/bench_emitter_sampler.py.  A step is one emitter_sample call
    (host term decomposition, one pe_emitter_weights launch per photon, host draws); the kernel roofline is
    against the live FP64 pipe peak; the CPU baseline runs the same matrix-cofactor sums in numpy
    (oracle/emitter_oracle.py) on a bounded sample of streams."""
    import math

    import numpy as np
    import torch

    from oracle import emitter_oracle as EO
    from photonic_engines_b200 import _native as NAT
    from photonic_engines_b200.clifford import emitter_sample
    from photonic_engines_b200.clifford.emitter import gap_terms
    from photonic_engines_b200.states import caterpillar, spin_gate

    n, m, shots = 12, 24, 512
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    st = caterpillar(n, [spin_gate(math.pi / 2, 0)] * n, m=m)
    g = torch.Generator().manual_seed(n)
    U_host = torch.linalg.qr(torch.randn(m, m, dtype=torch.complex128, generator=g))[0].contiguous()
    U = U_host.to(dev)
    peak = NAT.pipe_peak_tflops("f64", dev)
    for i in range(args.warmup):
        emitter_sample(st, U, shots, generator=torch.Generator().manual_seed(100 + i))
    torch.cuda.synchronize()
    kern_ms, flops = 0.0, 0.0
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        for i in range(args.steps):
            _, stats = emitter_sample(st, U, shots, generator=torch.Generator().manual_seed(i), return_stats=True)
            kern_ms += sum(stats["kernel_ms"])
            flops += sum(stats["flops"])
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    # end to end: U from pinned host memory every step, occupations back to the host
    U_pin = U_host.pin_memory()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for i in range(args.steps):
        occ = emitter_sample(st, U_pin.to(dev, non_blocking=True), shots, generator=torch.Generator().manual_seed(i))
        occ.cpu()
    e2e = args.steps * shots / (time.perf_counter() - t1)
    # CPU baseline: per stream and step, the pure terms and the numpy matrix-cofactor sums (16 streams)
    rng = np.random.default_rng(0)
    Un = U_host.numpy()
    t2 = time.perf_counter()
    nb = 16
    for _ in range(nb):
        order = rng.permutation(n)
        rows = []
        for k in range(1, n + 1):
            kept, s0, mats, f = gap_terms(st, order[:k].tolist(), torch.eye(2, dtype=torch.complex128)[0])
            colmode = np.array([list(st.modes[j]) for j in kept])
            w = EO.matrix_weights(Un, colmode, rows, s0.numpy(), mats.numpy(), f.numpy())
            rows.append(int(rng.choice(m, p=w / w.sum())))
    cpu = nb / (time.perf_counter() - t2)
    ach = flops / (kern_ms * 1e-3) / 1e12
    line = {"config": "emitter", "workload": f"EmitterMPS linear cluster (caterpillar), n={n} photons, m={m}, "
                                              f"chi=2, 2 labels, emitter traced, {shots} shots/step, Haar U",
            "metric": "samples/s", "unit": "samples/s", "value": args.steps * shots / dt,
            "ms_per_step": dt / args.steps * 1e3, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "dtype": "f64", "data": "synthetic", "kernel_share": kern_ms * 1e-3 / dt,
            "roofline": {"bound": "fp64", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                         "traffic": None, "flops_per_step": flops / args.steps,
                         "kernel_ms_per_step": kern_ms / args.steps},
            "e2e": {"value": e2e, "unit": "samples/s", "h2d_bytes_per_step": U_host.numel() * 16,
                    "d2h_bytes_per_step": shots * m * 8},
            "cpu_baseline": {"value": cpu, "unit": "samples/s", "cores": torch.get_num_threads(), "kind": "port",
                             "sample": f"{nb} streams, host pure terms + numpy matrix-cofactor sums per step"},
            "clocks": clk.summary(),
            "reference_gpu": None if args.no_reference_gpu else emitter_reference_leg(st, n, m, shots, U, args.steps)}
    print(json.dumps(line), flush=True)


def emitter_reference_leg(st, n: int, m: int, shots: int, U, steps: int) -> dict:
    """The same emitter workload through the reference's own emitter_sample (its default Triton backend,
    unmodified, from baseline/_ref) on this GPU: samples/s over `steps` calls after one untimed call, and how
    many occupation rows of the last call ours reproduces from the same generator seed."""
    import math

    import torch

    from photonic_engines_b200.clifford import emitter_sample
    ref = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref, "photonic_engines")):
        return {"unavailable": "baseline/_ref holds no install of the reference"}
    sys.path.insert(0, ref)
    try:
        import photonic_engines.clifford as rc
        from photonic_engines.states import EmitterMPS, spin_gate
    finally:
        sys.path.remove(ref)
    rst = EmitterMPS.caterpillar(n, [spin_gate(math.pi / 2, 0)] * n, m=m)
    try:
        rc.emitter_sample(rst, U, shots, generator=torch.Generator().manual_seed(100))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(steps):
            a = rc.emitter_sample(rst, U, shots, generator=torch.Generator().manual_seed(i))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    except Exception as e:                      # the reference's own code refusing this input or device
        return {"unavailable": f"{type(e).__name__}: {str(e)[:200]}"}
    b = emitter_sample(st, U, shots, generator=torch.Generator().manual_seed(steps - 1))
    same = int((a.cpu() == b.cpu()).all(dim=1).sum()) if a.shape == b.shape else 0
    return {"value": steps * shots / dt, "unit": "samples/s", "ms_per_call": dt / steps * 1e3,
            "identical_rows": same, "rows": int(a.shape[0]),
            "engine": "reference photonic_engines.clifford.emitter_sample, backend triton (its default)"}


def run_latency_and_adaptive(args):
    """`--config single`: one sample of the C2 workload (n = 20, m = 400) per fock_sample call — the latency
    path (the reference's single.py: one stream spread over the GPU, here the split steps), ms per sample,
    FP64 and mixed.  `--config adaptive`: the C2 workload with a forced prefix of 2 photons on modes (0, 1)
    and those modes avoided afterwards (adaptive optics), 2 000 shots per call: surviving samples/s and
    chains/s.  Both through the public fock_sample, U resident on the device."""
    import torch

    from photonic_engines_b200.clifford import fock_sample

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = torch.Generator().manual_seed(USEED)
    z = torch.randn(M_MODES, M_MODES, generator=g, dtype=torch.float64) + 1j * torch.randn(
        M_MODES, M_MODES, generator=g, dtype=torch.float64)
    q, r = torch.linalg.qr(z)
    d = torch.diagonal(r)
    U = (q * (d / d.abs()).unsqueeze(0)).to(dev)
    in_modes = list(range(N_PHOT))
    out = {}
    for precision in ("f64", "mixed"):
        gen = torch.Generator(device=dev).manual_seed(11)
        if args.config == "single":
            kw, shots = {}, 1
        else:
            kw, shots = {"prefix": [0, 1], "avoid": [0, 1], "keep_ids": True}, SHOTS
        for _ in range(args.warmup):
            fock_sample(U, in_modes, shots, generator=gen, precision=precision, **kw)
        torch.cuda.synchronize()
        kept = 0
        with ClockSampler(0) as clk:
            t0 = time.perf_counter()
            for _ in range(args.steps):
                res = fock_sample(U, in_modes, shots, generator=gen, precision=precision, **kw)
                if args.config == "adaptive":
                    kept += int(res[1].numel())
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
        if args.config == "single":
            out[precision] = {"ms_per_sample": dt / args.steps * 1e3, "samples_per_s": args.steps / dt,
                              "clocks": clk.summary()}
        else:
            out[precision] = {"chains_per_s": args.steps * shots / dt, "survivors_per_s": kept / dt,
                              "survival": kept / (args.steps * shots), "ms_per_step": dt / args.steps * 1e3,
                              "clocks": clk.summary()}
    # the same calls through the reference's own engine (Triton backend) on this GPU, beside ours in FP64
    ref_gpu = None
    if not args.no_reference_gpu:
        if args.config == "single":
            ref_gpu = public_call_leg([(U, in_modes)], 1, reps=args.steps)
        else:
            ref_gpu = public_call_leg([(U, in_modes)], SHOTS, reps=max(1, args.steps // 2),
                                      extra={"prefix": [0, 1], "avoid": [0, 1], "keep_ids": True})
    if args.config == "single":
        line = {"config": "single", "workload": WORKLOAD.replace("2000 shots/step", "1 shot per call"),
                "metric": "ms per sample (latency)", "unit": "ms", "value": out["f64"]["ms_per_sample"],
                "higher_is_better": False, "fp64": out["f64"], "mixed": out["mixed"], "n_gpus": 1,
                "steps": args.steps, "warmup": args.warmup, "data": "synthetic", "reference_gpu": ref_gpu}
    else:
        line = {"config": "adaptive", "workload": WORKLOAD + ", prefix (0, 1), avoid (0, 1)",
                "metric": "surviving samples/s", "unit": "samples/s", "value": out["mixed"]["survivors_per_s"],
                "higher_is_better": True, "fp64": out["f64"], "mixed": out["mixed"], "n_gpus": 1,
                "steps": args.steps, "warmup": args.warmup, "data": "synthetic", "reference_gpu": ref_gpu}
    print(json.dumps(line), flush=True)


# The reference's published FP64 numbers on one H100 PCIe for workloads of this path (production
# configuration): (label, n, m, shots per call, loss, published value, unit, source in the reference)
PUBLISHED = [
    ("s/sample n=24 m=2n", 24, 48, 2048, None, 0.35e-3, "s/sample", "docs/ALGORITHMS.md:186-194"),
    ("s/sample n=28 m=2n", 28, 56, 256, None, 1.9e-3, "s/sample", "docs/ALGORITHMS.md:186-194"),
    ("s/sample n=32 m=2n", 32, 64, 32, None, 22e-3, "s/sample", "docs/ALGORITHMS.md:186-194"),
    ("s/sample n=34 m=2n", 34, 68, 16, None, 69e-3, "s/sample", "docs/ALGORITHMS.md:186-194"),
    ("s/sample n=36 m=2n", 36, 72, 8, None, 0.23, "s/sample", "docs/ALGORITHMS.md:186-194"),
    ("s/sample n=38 m=2n", 38, 76, 4, None, 0.84, "s/sample", "docs/ALGORITHMS.md:186-194"),
    ("s/sample n=40 m=2n", 40, 80, 4, None, 2.6, "s/sample", "docs/ALGORITHMS.md:186-194"),
    ("samples/s k=6 m=12 plateau", 6, 12, 65536, None, 45.3e6, "samples/s", "results/keep/cost_table_20261011_h100.csv"),
    ("samples/s k=20 m=24", 20, 24, 4096, None, 108.0e3, "samples/s", "results/keep/cost_table_20261011_h100.csv"),
    ("samples/s k=20 m=32", 20, 32, 4096, None, 74.6e3, "samples/s", "results/keep/cost_table_20261011_h100.csv"),
    ("samples/s k=20 m=48", 20, 48, 4096, None, 45.1e3, "samples/s", "results/keep/cost_table_20261011_h100.csv"),
    ("samples/s k=20 m=96", 20, 96, 4096, None, 25.5e3, "samples/s", "results/keep/cost_table_20261011_h100.csv"),
    ("samples/s k=28 m=96", 28, 96, 256, None, 248.0, "samples/s", "results/keep/cost_table_20261011_h100.csv"),
    ("samples/s k=30 m=96", 30, 96, 64, None, 70.5, "samples/s", "results/keep/cost_table_20261011_h100.csv"),
    ("samples/s n=27 m=324", 27, 324, 256, None, 178.0, "samples/s", "results/keep/frontier3_fock_r12_20260920_h100.csv"),
    ("samples/s n=30 m=360", 30, 360, 64, None, 21.4, "samples/s", "results/keep/frontier3_fock_r12_20260920_h100.csv"),
    ("ms/sample lossy n=24 m=48 eta=1", 24, 48, 4096, 1.0, 0.54, "ms/sample", "docs/LOSS.md:93-95"),
    ("ms/sample lossy n=24 m=48 eta=0.9", 24, 48, 4096, 0.9, 0.22, "ms/sample", "docs/LOSS.md:93-95"),
    ("ms/sample lossy n=24 m=48 eta=0.7", 24, 48, 4096, 0.7, 0.056, "ms/sample", "docs/LOSS.md:93-95"),
    ("ms/sample lossy n=24 m=48 eta=0.5", 24, 48, 4096, 0.5, 0.034, "ms/sample", "docs/LOSS.md:93-95"),
    ("ms/sample lossy n=20 m=40 eta=1", 20, 40, 4096, 1.0, 0.051, "ms/sample", "results/keep/bench_loss_h100.csv:10-17"),
    ("ms/sample lossy n=20 m=40 eta=0.9", 20, 40, 4096, 0.9, 0.037, "ms/sample", "results/keep/bench_loss_h100.csv:10-17"),
    ("ms/sample lossy n=20 m=40 eta=0.7", 20, 40, 4096, 0.7, 0.030, "ms/sample", "results/keep/bench_loss_h100.csv:10-17"),
    ("ms/sample lossy n=20 m=40 eta=0.5", 20, 40, 4096, 0.5, 0.021, "ms/sample", "results/keep/bench_loss_h100.csv:10-17"),
]
PUBLISHED_ADDENDS = {24: 3.5e9, 28: 6.6e9, 32: 6.1e9}          # G addends/s, docs/ALGORITHMS.md:277-284


def run_published(args):
    """`--config published`: the workloads of the reference's published H100 numbers, run here through the
    public fock_sample (FP64, photons in modes 0..n-1, seeded Haar U, CUDA generator), one line with this
    GPU's figure, the published one and their ratio (> 1: faster here), frontier rows up to 40 photons
    included; beside them the reference's own engine (its fock_sample, Triton backend, from baseline/_ref)
    on this GPU for the same call, and how many of its occupation rows ours reproduces."""
    import numpy as np
    import torch

    from photonic_engines_b200.clifford import fock_sample
    from photonic_engines_b200.clifford.work import chain_work

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ref_fn, ref_why = (None, "skipped (--no-reference-gpu)") if args.no_reference_gpu else _reference_fock_sample()
    rows_out = []
    for label, n, m, shots, loss, pub, unit, src in PUBLISHED:
        g = torch.Generator().manual_seed(1000 + n + m)
        z = torch.randn(m, m, generator=g, dtype=torch.float64) + 1j * torch.randn(m, m, generator=g, dtype=torch.float64)
        q, r = torch.linalg.qr(z)
        d = torch.diagonal(r)
        U = (q * (d / d.abs()).unsqueeze(0)).to(dev)
        gen = torch.Generator(device=dev).manual_seed(5)
        kw = {} if loss is None else {"loss": loss}
        fock_sample(U, list(range(n)), shots, generator=gen, **kw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fock_sample(U, list(range(n)), shots, generator=gen, **kw)     # second warm call, timed: sizes reps
        torch.cuda.synchronize()
        reps = max(1, args.steps // 2, int(0.3 / max(time.perf_counter() - t0, 1e-6)))   # >= ~0.3 s per row
        t0 = time.perf_counter()
        for _ in range(reps):
            fock_sample(U, list(range(n)), shots, generator=gen, **kw)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / (reps * shots)               # seconds per sample
        here = {"s/sample": dt, "ms/sample": dt * 1e3, "samples/s": 1.0 / dt}[unit]
        ratio = pub / here if unit != "samples/s" else here / pub
        row = {"workload": label, "n": n, "m": m, "shots": shots, "loss": loss, "here": here, "published_h100": pub,
               "unit": unit, "speedup_vs_h100": ratio, "source": src}
        if loss is None and n in PUBLISHED_ADDENDS and label.startswith("s/sample"):
            # addends per sample from the rows of one call (the chain's exact term counts)
            from photonic_engines_b200.clifford import sample_chains
            sig = torch.argsort(torch.rand(min(shots, 64), n, generator=gen, device=dev), dim=1)
            res = sample_chains(U, list(range(n)), sig, seeds=torch.randint(0, 2 ** 31 - 1, (n,), device=dev),
                                split=None)
            add = chain_work(res["rows"].cpu().numpy(), m)["addends"] / sig.shape[0]
            row.update(addends_per_sample=add, g_addends_per_s=add / dt / 1e9,
                       published_g_addends_per_s=PUBLISHED_ADDENDS[n] / 1e9)
        if ref_fn is None:
            row["reference_b200"] = {"unavailable": ref_why}
        else:
            # the reference's own engine (Triton backend) on this GPU, the same call; shots cut so that one
            # call stays near 20 s at four times the published H100 time per sample
            pub_s = {"s/sample": pub, "ms/sample": pub * 1e-3, "samples/s": 1.0 / pub}[unit]
            ref_shots = shots if 4 * pub_s * shots <= 20 else max(1, int(20 / (4 * pub_s)))
            ref_fn(U, list(range(n)), 1, generator=torch.Generator(device=dev).manual_seed(3), **kw)  # builds kernels
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            a = ref_fn(U, list(range(n)), ref_shots, generator=torch.Generator(device=dev).manual_seed(11), **kw)
            torch.cuda.synchronize()
            dt_ref = (time.perf_counter() - t0) / ref_shots
            b = fock_sample(U, list(range(n)), ref_shots, generator=torch.Generator(device=dev).manual_seed(11), **kw)
            same = int((a.cpu() == b.cpu()).all(dim=1).sum())
            row["reference_b200"] = {"value": {"s/sample": dt_ref, "ms/sample": dt_ref * 1e3, "samples/s": 1.0 / dt_ref}[unit],
                                     "unit": unit, "shots": ref_shots, "identical_rows": same,
                                     "engine": "reference photonic_engines.clifford.fock_sample, backend triton"}
            row["speedup_vs_reference_b200"] = dt_ref / dt
        rows_out.append(row)
        print(json.dumps(row), file=sys.stderr, flush=True)
    line = {"config": "published", "metric": "speed-up over the reference's published H100 numbers (same workloads)",
            "unit": "x", "value": float(np.exp(np.mean([np.log(r_["speedup_vs_h100"]) for r_ in rows_out]))),
            "higher_is_better": True, "dtype": "f64", "data": "synthetic", "n_gpus": 1, "rows": rows_out,
            "note": "geometric mean of the per-row ratios"}
    on_b200 = [r_["speedup_vs_reference_b200"] for r_ in rows_out if "speedup_vs_reference_b200" in r_]
    if on_b200:
        line["speedup_vs_reference_b200_geomean"] = float(np.exp(np.mean(np.log(on_b200))))
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--ref-shots", type=int, default=0, help="chains per CPU sample (0: scaled to the cores)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU engine (baseline/_ref, Triton) on the same calls")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the c3 / c4 / c5 results the default line carries under 'configs'")
    ap.add_argument("--config", choices=("c1", "c2", "c3", "c4", "c5", "emitter", "single", "adaptive", "published"),
                    default="c2",
                    help="c2 (default) is the headline line; c1 c3 c4 c5 run through the batched sampler, emitter "
                         "the EmitterMPS path, single the one-sample latency path, adaptive prefix / avoid, published "
                         "the workloads of the reference's published H100 numbers")
    ap.add_argument("--profile-batch", choices=("c1", "c3", "c4", "c5"), default=None,
                    help="run only five eager FP64 batches of a configuration (a target for an ncu launch list)")
    ap.add_argument("--profile-launch", choices=FORMS, default=None,
                    help="run only two chain launches of the workload (a target for ncu -s 1 -c 1)")
    args = ap.parse_args()
    if args.profile_batch:
        profile_batch(args.profile_batch)
        return
    if args.profile_launch:
        profile_launch(args.profile_launch)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.config == "emitter" and args.impl == "b200":
        run_emitter(args)
        return
    if args.config == "published" and args.impl == "b200":
        run_published(args)
        return
    if args.config in ("single", "adaptive") and args.impl == "b200":
        run_latency_and_adaptive(args)
        return
    if args.config != "c2" and args.impl == "b200":
        run_config(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
