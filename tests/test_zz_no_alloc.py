"""The allocation-free chain entry point (pe_fock_chain_noalloc) against the regular one (pe_fock_chain).

pe_fock_chain_noalloc serves callers that cannot allocate device memory when they sample — a host
callback, a serving process whose device memory all belongs to its own arena, a foreign-language binding
that can pass buffers but not call cudaMalloc.  It keeps the chain kernel's scratch (work-queue counter
and status word) in a static device array instead of a caller-provided workspace.  Both entry points are
called here through the C ABI (ctypes) on the same inputs; the allocation-free one twice in a row (the
array keeps the previous call's contents, so the second call checks that each call clears it).  Rows and
occupations must match exactly, marginals within the FP64 tolerance of the parity tests (1e-10 relative).

This file is named to be collected last, so that a run stopping at the first failure has already run
every other test; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

from photonic_engines_b200 import _native as N
from photonic_engines_b200.clifford.kernels import pack_instances

pytestmark = pytest.mark.gpu
F64_TOL = 1e-10


def _haar(m, seed):
    g = torch.Generator().manual_seed(seed)
    z = torch.randn(m, m, generator=g, dtype=torch.float64) + 1j * torch.randn(m, m, generator=g, dtype=torch.float64)
    q, r = torch.linalg.qr(z)
    d = torch.diagonal(r)
    return q * (d / d.abs()).unsqueeze(0)


def _inputs(n, m, S, seed):
    dev = torch.device("cuda")
    U = _haar(m, seed).to(dev)
    acol, off, mm, nn = pack_instances(U, list(range(n)))
    g = torch.Generator(device=dev).manual_seed(seed)
    cols = torch.argsort(torch.rand(S, n, generator=g, device=dev), dim=1).contiguous()
    seeds = torch.randint(0, 2 ** 31 - 1, (1, n), generator=g, device=dev).contiguous()
    dp = torch.zeros(S, dtype=torch.int64, device=dev)
    return torch.view_as_real(acol).contiguous(), off, mm, nn, dp, cols, seeds


def _outputs(S, n, m):
    dev = torch.device("cuda")
    return (torch.full((S, n), -1, dtype=torch.int64, device=dev), torch.full((S, m), -1, dtype=torch.int64, device=dev),
            torch.zeros(S, n, m, dtype=torch.float64, device=dev))


@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("n,m,S", [(6, 12, 64), (14, 60, 48)])
def test_noalloc_entry_point_matches_the_regular_one(precision, n, m, S):
    L = N.load()
    a, off, mm, nn, dp, cols, seeds = _inputs(n, m, S, 17 + n)
    stream = N.stream_handle(a.device)
    prec = N.PRECISIONS[precision]
    ws = N.workspace(a.device)
    rows0, occ0, marg0 = _outputs(S, n, m)
    rc = L.pe_fock_chain(prec, a.data_ptr(), off.data_ptr(), mm.data_ptr(), nn.data_ptr(), 1, m, S, dp.data_ptr(),
                         None, cols.data_ptr(), n, None, seeds.data_ptr(), None, None, None, rows0.data_ptr(),
                         occ0.data_ptr(), m, marg0.data_ptr(), m, ws.data_ptr(), ws.numel(), 0, 0, 0, stream)
    assert rc == 0, L.pe_status_string(rc).decode()
    for call in range(2):
        rows, occ, marg = _outputs(S, n, m)
        status = torch.full((1,), 123, dtype=torch.int32, device=a.device)
        rc = L.pe_fock_chain_noalloc(prec, a.data_ptr(), off.data_ptr(), mm.data_ptr(), nn.data_ptr(), 1, m, S,
                                     dp.data_ptr(), None, cols.data_ptr(), n, None, seeds.data_ptr(), None, None, None,
                                     rows.data_ptr(), occ.data_ptr(), m, marg.data_ptr(), m, status.data_ptr(), 0, 0, 0,
                                     stream)
        assert rc == 0, L.pe_status_string(rc).decode()
        torch.cuda.synchronize()
        assert int(status.item()) == 0, f"call {call}: device status {int(status.item())}"
        assert torch.equal(rows, rows0), f"call {call}: rows differ"
        assert torch.equal(occ, occ0), f"call {call}: occupations differ"
        rel = ((marg - marg0).abs().amax(dim=2) / marg0.abs().amax(dim=2)).max().item()
        assert rel <= F64_TOL, f"call {call}: marginal difference {rel:.2e}"
    st, _ = N.read_status(ws)
    assert st == 0


def test_noalloc_entry_point_reports_argument_errors_like_the_regular_one():
    L = N.load()
    a, off, mm, nn, dp, cols, seeds = _inputs(4, 8, 4, 3)
    rows, occ, marg = _outputs(4, 4, 8)
    rc = L.pe_fock_chain_noalloc(7, a.data_ptr(), off.data_ptr(), mm.data_ptr(), nn.data_ptr(), 1, 8, 4, dp.data_ptr(),
                                 None, cols.data_ptr(), 4, None, seeds.data_ptr(), None, None, None, rows.data_ptr(),
                                 occ.data_ptr(), 8, None, 8, None, 0, 0, 0, N.stream_handle(a.device))
    assert rc == N.load().pe_fock_chain(7, None, None, None, None, 1, 8, 4, None, None, None, 4, None, None, None, None,
                                        None, None, None, 8, None, 8, None, 0, 0, 0, 0, None)
    assert ctypes.c_int(rc).value < 0
