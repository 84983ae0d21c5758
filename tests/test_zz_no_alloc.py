"""pfsf_compact_failures_noalloc: the allocation-free failure compaction.

Some callers cannot call cudaMalloc (a physics thread that must not absorb
the device-wide synchronisation allocation can cause inside its tick budget,
or code that only borrows device buffers).  For them the library offers a
failure compaction whose scratch lives in a fixed array inside the library.
This test drives it through the C ABI with caller-owned device buffers and
checks that two calls in a row each reproduce, bit for bit (integer data),
the failure buffer pfsf_tick_dbb produced for the same failure flags.  It
runs last in the suite (file name) and also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

import cases
from pfsf_b200 import capi

pytestmark = pytest.mark.gpu


def test_noalloc_compaction_matches_tick_failure_buffer(lib_built):
    import torch

    cfg = capi.default_config(max_island_size=1 << 24, tick_budget_ms=1 << 30)
    eng = capi.Engine(cfg)
    assert eng.init() == capi.PFSF_OK, "CUDA device required"
    case = cases.compat_case("noise20")
    case["rcomp"][::3] = 1e-9  # make a good share of the voxels fail
    origin = (40, -7, 12)
    iid = 9001
    assert eng.add_island(iid, case["dims"], origin) == capi.PFSF_OK
    host = {k: case[k].copy() for k in ("phi", "source", "conductivity", "type", "rcomp", "rtens", "max_phi")}
    assert eng.register_buffers(iid, host["phi"], host["source"], host["conductivity"], host["type"],
                                host["rcomp"], host["rtens"], host["max_phi"]) == capi.PFSF_OK
    cap = 4096
    fb = np.zeros(1 + 4 * cap, np.int32)
    assert eng.tick_dbb([iid], fb) == capi.PFSF_OK
    count = int(fb[0])
    assert 0 < count < cap
    flags = eng.debug_field(iid, 3)

    dev = torch.device("cuda", 0)
    d_fail = torch.from_numpy(flags).to(dev)
    d_tuples = torch.empty(4 * cap, dtype=torch.int32, device=dev)
    d_count = torch.empty(1, dtype=torch.int32, device=dev)
    lx, ly, lz = case["dims"]
    for rep in range(2):
        d_tuples.fill_(-7)
        d_count.fill_(-1)
        torch.cuda.synchronize()
        rc = eng.L.pfsf_compact_failures_noalloc(C.c_void_p(d_fail.data_ptr()), lx, ly, lz, capi.Pos(*origin),
                                                 C.c_void_p(d_tuples.data_ptr()), cap,
                                                 C.c_void_p(d_count.data_ptr()), None)
        assert rc == capi.PFSF_OK
        torch.cuda.synchronize()
        got_count = int(d_count.cpu().item())
        got = d_tuples.cpu().numpy()
        assert got_count == count, f"call {rep}: count {got_count} vs {count}"
        np.testing.assert_array_equal(got[: 4 * count], fb[1: 1 + 4 * count])
        assert np.all(got[4 * count:] == -7)

    # a buffer smaller than the failure count: *dev_count is still the full
    # count, the first `small` tuples are written, nothing past them; on a
    # non-default stream the caller orders its reads after the stream
    small = count // 3
    assert small > 0
    side = torch.cuda.Stream(device=dev)
    for rep in range(2):
        d_tuples.fill_(-7)
        d_count.fill_(-1)
        torch.cuda.synchronize()
        rc = eng.L.pfsf_compact_failures_noalloc(C.c_void_p(d_fail.data_ptr()), lx, ly, lz, capi.Pos(*origin),
                                                 C.c_void_p(d_tuples.data_ptr()), small,
                                                 C.c_void_p(d_count.data_ptr()), C.c_void_p(side.cuda_stream))
        assert rc == capi.PFSF_OK
        side.synchronize()
        assert int(d_count.cpu().item()) == count
        got = d_tuples.cpu().numpy()
        np.testing.assert_array_equal(got[: 4 * small], fb[1: 1 + 4 * small])
        assert np.all(got[4 * small:] == -7), f"call {rep}: tuples written past the capacity"

    # sizes beyond the fixed scratch are rejected, nothing is launched
    rc = eng.L.pfsf_compact_failures_noalloc(C.c_void_p(d_fail.data_ptr()), 4096, 4096, 8, capi.Pos(0, 0, 0),
                                             C.c_void_p(d_tuples.data_ptr()), cap, C.c_void_p(d_count.data_ptr()),
                                             None)
    assert rc == capi.PFSF_ERROR_INVALID_ARG
    eng.close()
