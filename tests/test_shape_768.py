"""The 10M x 768 configuration's shape at a size the oracle checks in seconds:
d = 768, K = 16,384 clusters of Zipf-distributed sizes (every cluster
non-empty), total bits 3, 5 and 9 (EX = 2, 4, 8).  K above 4,096 takes the
probe's unstaged key path and its larger sort buffers; D = 768 gives 12
64-dimension chunks.  The GPU search must equal the C oracle bit for bit
(ids and distances), and the batched plan must equal the per-query search."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

K, DIM, N, NQ = 16384, 768, 131072, 48


@pytest.fixture(scope="module")
def shape768(tmp_path_factory):
    rng = np.random.default_rng(768)
    # cluster sizes: one vector each, the rest Zipf(1.1)-distributed
    w = 1.0 / np.arange(1, K + 1) ** 1.1
    ids = np.concatenate([np.arange(K), rng.choice(K, size=N - K, p=w / w.sum())])
    rng.shuffle(ids)
    centres = rng.standard_normal((K, DIM)).astype(np.float32)
    centres /= np.linalg.norm(centres, axis=1, keepdims=True)
    base = centres[ids] + 0.05 * rng.standard_normal((N, DIM)).astype(np.float32)
    qc = rng.choice(K, size=NQ, p=w / w.sum())
    query = centres[qc] + 0.05 * rng.standard_normal((NQ, DIM)).astype(np.float32)
    sums = torch.zeros(K, DIM, dtype=torch.float64).index_add_(
        0, torch.from_numpy(ids.astype(np.int64)), torch.from_numpy(base).double())
    cent = (sums / torch.from_numpy(np.bincount(ids, minlength=K))[:, None]).float().numpy()
    return tmp_path_factory.mktemp("shape768"), base, cent, ids, query


@pytest.mark.parametrize("bits", [3, 5, 9])
def test_search_equals_oracle(shape768, bits, oracle_mod):
    from erq_b200 import IVF, Plan, build_index, indexfile

    d, base, cent, ids, query = shape768
    arr = build_index.build_index_torch(torch.from_numpy(base).cuda(), torch.from_numpy(cent).cuda(),
                                        torch.from_numpy(ids.astype(np.int64)).cuda(), bits,
                                        seed=bits)
    path = os.path.join(d, f"b{bits}.index")
    indexfile.write_index(path, arr)
    idx = IVF(path)
    assert (idx.K, idx.DIM, idx.D, idx.EX_BITS) == (K, DIM, DIM, bits - 1)
    qr = idx.rotate(query)
    o = oracle_mod.Oracle(path)
    for k, nprobe in ((100, 64), (10, 200)):
        got_ids, got_d = idx.search_batch(qr, k, nprobe)
        ref_ids, ref_d = o.search(qr, k, nprobe, nthreads=8)
        assert (got_ids == ref_ids).all(), (bits, k, nprobe)
        assert (got_d.view(np.uint32) == ref_d.view(np.uint32)).all(), (bits, k, nprobe)
    o.close()
    # the batched plan (work-list scan, graph replay) on the same queries
    ref_ids, ref_d = idx.search_batch(qr, 100, 64)
    plan = Plan(idx, max_batch=NQ, k=100, nprobe=64)
    for _ in range(2):
        p_ids, p_d, _ = plan.search(qr)
        assert (p_ids == ref_ids).all()
        assert (p_d.view(np.uint32) == ref_d.view(np.uint32)).all()
    plan.free()
    idx.free()
