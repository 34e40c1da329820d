"""The no-allocation entry point mb_k2_plain_noalloc_dev.

It serves callers that cannot allocate device memory (host callbacks, fixed memory budgets,
runtimes that own every allocation): the test allocates all buffers itself (with torch, as
such a caller's runtime would) and the entry point only reads and writes them, keeping its
partial sums in the library's fixed device array.  Its results must match the table-based
plain entry point on two calls in a row.  This file is collected last so that a run which
stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from mertens_bound_b200 import _lib, k2, synth

pytestmark = pytest.mark.gpu


def _device_arrays(torch, data, dev):
    n = data.n
    G3 = data.G3
    limbs = np.stack([G3[:, 2] & 0xFFFFFFFF, G3[:, 2] >> 32, G3[:, 1] & 0xFFFFFFFF, G3[:, 1] >> 32,
                      G3[:, 0]]).astype(np.uint32)
    g = torch.from_numpy(limbs.reshape(-1).view(np.int32).copy()).to(dev)
    gam = torch.from_numpy(data.gamma.copy()).to(dev)
    cre = torch.from_numpy(data.c_re.copy()).to(dev)
    cim = torch.from_numpy(data.c_im.copy()).to(dev)
    return n, g, gam, cre, cim


def _call(L, arrs, n_use, cd_dev, P, k, out, stream):
    n, g, gam, cre, cim = arrs
    vi, vf, dl = cd_dev
    return L.mb_k2_plain_noalloc_dev(g.data_ptr(), gam.data_ptr(), cre.data_ptr(), cim.data_ptr(), n, n_use, P,
                                     vi.data_ptr(), vf.data_ptr(), dl.data_ptr(), k,
                                     out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), stream)


def _cand_dev(torch, cd, dev):
    return (torch.from_numpy(cd.v_int.view(np.int64).copy()).to(dev),
            torch.from_numpy(cd.v_frac.view(np.int64).copy()).to(dev),
            torch.from_numpy(cd.delta.copy()).to(dev))


def test_noalloc_matches_table_entry_point(gpu, oracle):
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    data = synth.make_table(20_000, seed=5)
    cd = synth.make_candidates(300, seed=6)
    cd.delta[:] = np.linspace(-1e-4, 1e-4, cd.n)
    k, T = 3e-9, 15_000.0
    with k2.ZeroTable.from_data(data) as t:
        rv, rd, rk = k2.k2_plain(t, cd, k, T)
    n_use = data.count_below(T)
    arrs = _device_arrays(torch, data, dev)
    cdd = _cand_dev(torch, cd, dev)
    out = torch.empty(3, cd.n, dtype=torch.float64, device=dev)
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    ohi, _ = oracle.k2(cd.subset(np.arange(16)), data, k, n_use)
    for _ in range(2):                                   # two calls in a row share the scratch
        out.fill_(float("nan"))
        st = _call(L, arrs, n_use, cdd, cd.n, k, out, stream)
        assert st == 0, L.mb_last_error()
        torch.cuda.synchronize(dev)
        v, d, kk = (out[i].cpu().numpy() for i in range(3))
        # the same kernels with the same shape and chunk count as the table-based entry point:
        # the same bits
        assert np.array_equal(v, rv) and np.array_equal(d, rd) and np.array_equal(kk, rk)
        # and the plain kernel's tolerance against the binary128 oracle
        assert np.max(np.abs(v[:16] - ohi[:, 0])) < 2e-13
        assert np.max(np.abs(d[:16] - ohi[:, 1])) < 2e-13 * np.max(np.abs(ohi[:, 1]))
        assert np.max(np.abs(kk[:16] - ohi[:, 2])) < 2e-13 * np.max(np.abs(ohi[:, 2]))


def test_noalloc_fewer_chunks_at_large_p(gpu):
    """At P = 200,000 the fixed array holds one chunk of partial sums where the table-based entry
    point uses more: the zero sums are split differently, so the results agree to rounding."""
    import torch

    dev = torch.device("cuda", 0)
    data = synth.make_table(12_000, seed=7)
    cd = synth.make_candidates(200_000, seed=8)
    k = 3e-9
    with k2.ZeroTable.from_data(data) as t:
        rv, rd, rk = k2.k2_plain(t, cd, k)
    arrs = _device_arrays(torch, data, dev)
    cdd = _cand_dev(torch, cd, dev)
    out = torch.empty(3, cd.n, dtype=torch.float64, device=dev)
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(2):
        out.fill_(float("nan"))
        assert _call(L, arrs, data.n, cdd, cd.n, k, out, stream) == 0, L.mb_last_error()
        torch.cuda.synchronize(dev)
        v, d, kk = (out[i].cpu().numpy() for i in range(3))
        assert np.max(np.abs(v - rv)) < 2e-13
        assert np.max(np.abs(d - rd)) < 2e-13 * np.max(np.abs(rd))
        assert np.max(np.abs(kk - rk)) < 2e-13 * np.max(np.abs(rk))


def test_noalloc_rejects_oversize(gpu):
    L = _lib.lib()
    st = L.mb_k2_plain_noalloc_dev(None, None, None, None, 1, 1, 400_000, None, None, None, 3e-9,
                                   None, None, None, None)
    assert st == -6 and b"exceeds the fixed scratch" in L.mb_last_error()      # MB_ERR_CAPACITY
    st = L.mb_k2_plain_noalloc_dev(None, None, None, None, 1, 1, -1, None, None, None, 3e-9,
                                   None, None, None, None)
    assert st == -1                                                            # MB_ERR_ARG
