"""mgc_row_offsets_static: CSR row offsets of a device-resident synapse list
computed with the library's static scratch array (no allocation) equal the
row_ptr that mgc_create builds for the same list (read back with
mgc_export_csr), on two calls in a row.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import mgbrain_b200 as mgb
from mgbrain_b200 import brunel, capi


def row_offsets_static(src_d, n, out_d, stream):
    return capi.lib().mgc_row_offsets_static(C.c_void_p(src_d.data_ptr()), src_d.numel(), n,
                                             C.c_void_p(out_d.data_ptr()), C.c_void_p(stream))


def network(n, S, seed):
    """Random LIF0 network (never fires): only the synapse list matters here.
    Sources are skewed so some rows are empty and some long."""
    rng = np.random.default_rng(seed)
    src = (n * rng.random(S) ** 2).astype(np.int32)
    tar = rng.integers(0, n, S).astype(np.int32)
    w = np.full(S, 1e-4, np.float32)
    d = rng.integers(1, 4, S).astype(np.int32)
    return src, tar, w, d


@pytest.mark.gpu
@pytest.mark.parametrize("n,S", [(1, 0), (4095, 1), (10_000, 200_000), (300_001, 1_500_000)])
def test_static_row_offsets_equal_create(n, S):
    import torch
    src, tar, w, d = network(n, S, seed=n)
    types = np.full(n, mgb.LIF0, np.int8)
    if S:
        sim = mgb.Simulator.from_arrays(n, types, src, tar, w, d, brunel.brunel_lifconst(),
                                        mode=mgb.MODE_PUSH)
        expect = sim.export_csr()[0]
        sim.close()
    else:
        expect = np.zeros(n + 1, np.int64)
    assert expect[-1] == S
    src_d = torch.from_numpy(src).cuda()
    out_d = torch.full((n + 1,), -7, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        assert row_offsets_static(src_d, n, out_d, stream) == capi.MGC_OK, capi.lib().mgc_last_error()
        assert np.array_equal(out_d.cpu().numpy(), expect)
        out_d.fill_(123)   # the second call must overwrite everything


@pytest.mark.gpu
def test_static_row_offsets_allocate_nothing():
    """The library's allocation-failure injector is armed for the very next
    device allocation; two static calls still succeed, and the injected
    failure is still pending afterwards (the next builder meets it), so
    neither call allocated through the library."""
    import torch
    n, S = 50_000, 400_000
    src, _, _, _ = network(n, S, seed=3)
    src_d = torch.from_numpy(src).cuda()
    out_d = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    expect = np.concatenate([[0], np.cumsum(np.bincount(src, minlength=n))]).astype(np.int64)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    mgb.capi.fault_inject_alloc(1)
    try:
        for _ in range(2):
            assert row_offsets_static(src_d, n, out_d, stream) == capi.MGC_OK, capi.lib().mgc_last_error()
            assert np.array_equal(out_d.cpu().numpy(), expect)
        assert torch.cuda.mem_get_info()[0] >= free0 - (2 << 20)
        with pytest.raises(capi.MgcError) as e:   # the pending failure: this builder's first allocation
            mgb.Simulator.from_arrays(4, np.full(4, mgb.LIF0, np.int8), np.zeros(1, np.int32),
                                      np.ones(1, np.int32), np.ones(1, np.float32), np.ones(1, np.int32),
                                      brunel.brunel_lifconst())
        assert e.value.status == capi.MGC_ERR_NOMEM
    finally:
        mgb.capi.fault_inject_alloc(0)


@pytest.mark.gpu
def test_static_row_offsets_reject_bad_input():
    import torch
    out_d = torch.zeros(8, dtype=torch.int64, device="cuda")
    src_d = torch.tensor([0, 5, 9, 2], dtype=torch.int32, device="cuda")   # 9 is out of range for n=7
    stream = torch.cuda.current_stream().cuda_stream
    assert row_offsets_static(src_d, 7, out_d, stream) == capi.MGC_ERR_INVALID
    assert b"outside [0, 7)" in capi.lib().mgc_last_error()
    # beyond the static scratch: rejected before touching the device
    L = capi.lib()
    assert L.mgc_row_offsets_static(C.c_void_p(src_d.data_ptr()), 4, 200_000_000,
                                    C.c_void_p(out_d.data_ptr()), C.c_void_p(stream)) == capi.MGC_ERR_INVALID
    assert b"static scratch limit of 134217727" in L.mgc_last_error()
    # a good call right after the rejected ones
    src_ok = torch.tensor([0, 5, 6, 2, 5], dtype=torch.int32, device="cuda")
    assert row_offsets_static(src_ok, 7, out_d, stream) == capi.MGC_OK
    assert out_d.cpu().tolist() == [0, 1, 1, 2, 2, 2, 4, 5]
