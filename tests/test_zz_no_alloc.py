"""erq_search_noalloc: the search for callers that cannot allocate device memory.

Some callers own all GPU memory through their own allocator, or forbid any
allocation while a request is served; erq_search takes its scratch from a
memory pool and so does not suit them.  erq_search_noalloc runs the same
pipeline with its scratch in a fixed array inside the library.  These tests
call it through the C ABI and require results identical to erq_search's
(the suite's tolerance for the search is bit-exact) on two calls in a row,
the second reusing the array the first one left behind.  This file is named
to be collected last.
"""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _call(lib, idx, q, k, nprobe, ids, dists, stream):
    return lib.erq_search_noalloc(idx._h, C.c_void_p(q.data_ptr()), q.shape[0], k, nprobe,
                                  C.c_void_p(ids.data_ptr()),
                                  C.c_void_p(dists.data_ptr()) if dists is not None else None,
                                  C.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("name", ["d128_b4_mix", "d100_b8_edges"])
def test_noalloc_matches_search_on_two_calls(name):
    from erq_b200 import IVF, load_library

    lib = load_library()
    g = load_golden(name)
    k, nprobe = int(g["k"]), int(g["nprobe"])
    idx = IVF(g["path"])
    q = torch.from_numpy(g["qrot"]).cuda()
    stream = torch.cuda.current_stream()
    ref_ids, ref_d = idx.search_batch(q, k, nprobe, stream=stream)
    torch.cuda.synchronize()
    ref_ids = ref_ids.cpu().numpy()
    ref_d = ref_d.cpu().numpy()
    for _ in range(2):
        ids = torch.full((q.shape[0], k), -1, dtype=torch.int32, device="cuda")
        d = torch.full((q.shape[0], k), -1.0, dtype=torch.float32, device="cuda")
        assert _call(lib, idx, q, k, nprobe, ids, d, stream) == 0, lib.erq_last_error()
        torch.cuda.synchronize()
        assert (ids.cpu().numpy() == ref_ids).all()
        assert (d.cpu().numpy().view(np.uint32) == ref_d.view(np.uint32)).all()
    # and both equal the reference's own results for these bytes
    assert (ref_ids.view(np.uint32) == g["ids"]).all()
    idx.free()


def test_noalloc_rejects_what_it_cannot_hold():
    from erq_b200 import IVF, load_library

    lib = load_library()
    g = load_golden("d128_b4_mix")
    idx = IVF(g["path"])
    stream = torch.cuda.current_stream()
    nq = 200_000  # far beyond the fixed scratch for this index
    q = torch.zeros((nq, idx.D), dtype=torch.float32, device="cuda")
    ids = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
    assert _call(lib, idx, q, 10, idx.K, ids, None, stream) == 1
    msg = lib.erq_last_error().decode()
    assert "static scratch" in msg and "queries per call" in msg
    # the batch the message reports fits exactly: that many queries run and
    # equal erq_search, one more is refused
    fit = int(re.search(r"at most (\d+) queries per call", msg).group(1))
    assert 0 < fit < nq
    gen = torch.Generator().manual_seed(7)
    qf = torch.randn((fit + 1, idx.D), generator=gen, dtype=torch.float32).cuda()
    ids_f = torch.full((fit + 1, 10), -1, dtype=torch.int32, device="cuda")
    d_f = torch.full((fit + 1, 10), -1.0, dtype=torch.float32, device="cuda")
    assert _call(lib, idx, qf, 10, idx.K, ids_f, d_f, stream) == 1
    assert _call(lib, idx, qf[:fit], 10, idx.K, ids_f, d_f, stream) == 0, lib.erq_last_error()
    torch.cuda.synchronize()
    ref_ids, ref_d = idx.search_batch(qf[:fit], 10, idx.K, stream=stream)
    torch.cuda.synchronize()
    assert (ids_f[:fit].cpu().numpy() == ref_ids.cpu().numpy()).all()
    assert (d_f[:fit].cpu().numpy().view(np.uint32) == ref_d.cpu().numpy().view(np.uint32)).all()
    # host buffers are refused: copying them would need device memory
    qh = torch.zeros((4, idx.D), dtype=torch.float32)
    ih = torch.empty((4, 10), dtype=torch.int32)
    assert _call(lib, idx, qh, 10, 2, ih, None, stream) == 1
    assert "device memory only" in lib.erq_last_error().decode()
    idx.free()
