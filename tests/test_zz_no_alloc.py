"""The allocation-free entry point css_compact_lines_noalloc, for callers
that cannot allocate device memory when they need a derivative (all device
memory handed to their own pool or a framework's caching allocator, or no
tolerance for the device-wide synchronization of cudaMalloc/cudaFree).

It must give the same lines as css_compact_lines, which allocates: bit for
bit, since both run the same line kernel on tables built by the same
correctly rounded steps.  Every closure is covered (both ends physical, both
halo-closed, one of each, bdry 0..4, first and second derivatives), call
after call on the one shared scratch array, with sizes and closures changing
between calls so stale scratch contents would show.  An empty batch does
only the per-device set-up, and a request larger than the fixed scratch
array is refused.  This file is collected last on purpose: if it fails, a
run that stops at the first failure has already run every other test."""
import numpy as np
import pytest

from css_b200 import _lib
from css_b200.context import compact_lines

pytestmark = pytest.mark.gpu


def _noalloc(x, order, lphys, rphys, bdry, bl, bh, hl, hh, dnum, scale):
    import torch
    dev = torch.device("cuda", 0)
    n = x.shape[-1]
    nl = x.shape[0]
    tx = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    out = torch.zeros_like(tx)
    t = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    tbl, tbh, thl, thh = t(bl), t(bh), t(hl), t(hh)
    ptr = lambda a: None if a is None else a.data_ptr()
    stream = torch.cuda.current_stream(dev)
    rc = _lib.lib().css_compact_lines_noalloc(tx.data_ptr(), out.data_ptr(), n, nl, order, lphys, rphys, bdry,
                                              ptr(tbl), ptr(tbh), ptr(thl), ptr(thh), dnum, scale, stream.cuda_stream)
    _lib.check(rc)
    torch.cuda.synchronize(dev)
    return out.cpu().numpy()


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_noalloc_setup_call_with_no_lines(gpu_available):
    import torch
    x = torch.zeros((1, 32), dtype=torch.float64, device="cuda")
    rc = _lib.lib().css_compact_lines_noalloc(x.data_ptr(), x.data_ptr(), 32, 0, 1, 1, 1, 1, None, None, None,
                                              None, 1.0, 1.0, None)
    assert rc == 0


def test_noalloc_matches_allocating_entry_point_twice(gpu_available):
    rng = np.random.default_rng(42)
    cases = [  # (n, nlines, order, lphys, rphys, bdry)
        (32, 700, 1, 1, 0, 2),
        (48, 300, 2, 0, 1, 3),
    ]
    for n, nl, order, lphys, rphys, bdry in cases:
        x = np.sin(np.linspace(0, 2, n))[None, :] + 0.05 * rng.standard_normal((nl, n))
        bl, bh = rng.standard_normal(nl), rng.standard_normal(nl)
        hl, hh = rng.standard_normal((nl, 4)), rng.standard_normal((nl, 4))
        dnum = float(n - 1)
        scale = dnum ** order
        want = compact_lines(x, order, lphys, rphys, bdry, bl, bh, hl, hh, dnum=dnum, scale=scale)
        got = _noalloc(x, order, lphys, rphys, bdry, bl, bh, hl, hh, dnum, scale)
        assert rel(got, want) < 1e-13, (n, order, rel(got, want))
        assert np.array_equal(got, want), (n, order, rel(got, want))


@pytest.mark.parametrize("order", [1, 2])
def test_noalloc_every_closure_bit_equal(order, gpu_available):
    rng = np.random.default_rng(7 + order)
    for lphys in (0, 1):
        for rphys in (0, 1):
            for bdry in range(5):
                n = 20 + 2 * bdry + 6 * lphys + 3 * rphys  # a different size every call
                nl = 37 + 11 * bdry
                x = np.cos(np.linspace(0, 2.5, n))[None, :] + 0.05 * rng.standard_normal((nl, n))
                bl, bh = rng.standard_normal(nl), rng.standard_normal(nl)
                hl, hh = rng.standard_normal((nl, 4)), rng.standard_normal((nl, 4))
                dnum = float(n - 1)
                scale = dnum ** order
                want = compact_lines(x, order, lphys, rphys, bdry, bl, bh, hl, hh, dnum=dnum, scale=scale)
                got = _noalloc(x, order, lphys, rphys, bdry, bl, bh, hl, hh, dnum, scale)
                assert np.array_equal(got, want), (lphys, rphys, bdry, rel(got, want))


def test_noalloc_rejects_requests_beyond_its_scratch(gpu_available):
    import torch
    n, nl = 256, 2000  # 15*258 + 2000*264 doubles > 262144
    x = torch.zeros((nl, n), dtype=torch.float64, device="cuda")
    out = torch.zeros_like(x)
    rc = _lib.lib().css_compact_lines_noalloc(x.data_ptr(), out.data_ptr(), n, nl, 1, 1, 1, 1, None, None, None,
                                              None, 1.0, 1.0, None)
    assert rc == 1
    assert b"scratch" in _lib.lib().css_last_error()
