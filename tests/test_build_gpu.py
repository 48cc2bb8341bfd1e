"""Index construction on the GPU (erq_build_index, build.cuh) against the
reference's own create_index (src/create_index.cpp compiled by
oracle/Makefile) on the same data, centroids, cluster ids and rotation:
every byte of the file must be equal - header, cluster sizes, rotation,
rotated centroids, the 1-bit FastScan blocks with their factors, the EX-bit
codes (fast_quantize's exact sweep), xipnorm and ids - except the factors
of the lanes past a cluster's end, which the reference leaves unset."""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

CREATE_INDEX = os.path.join(REPO, "oracle", "_ref", "create_index")


def _reference_index(tmp_path, base, cent, ids, bits):
    from erq_b200 import vecs

    if not os.access(CREATE_INDEX, os.X_OK):
        pytest.skip("reference build (make -C oracle ref) not present")
    K = cent.shape[0]
    ds = "bld"
    ddir = tmp_path / "data" / ds
    ddir.mkdir(parents=True, exist_ok=True)
    (tmp_path / "bin").mkdir(exist_ok=True)
    (tmp_path / "results" / "indexing_time").mkdir(parents=True, exist_ok=True)
    vecs.write_vecs(str(ddir / f"{ds}_base.fvecs"), base)
    vecs.write_vecs(str(ddir / f"{ds}_centroid_{K}.fvecs"), cent)
    vecs.write_vecs(str(ddir / f"{ds}_cluster_id_{K}.ivecs"), ids.astype(np.int32)[:, None])
    subprocess.run([CREATE_INDEX, ds, str(K), str(bits)], cwd=tmp_path / "bin", check=True,
                   stdout=subprocess.DEVNULL, timeout=900)
    return str(ddir / f"ivf_exhaf{bits}.index")


def _case(n, dim, K, seed, sphere=False):
    from erq_b200 import datasets

    if sphere:
        base, _ = datasets.sphere_mixture(n, dim, 32, 0.05, seed=seed)
    else:
        base, _ = datasets.gaussian_mixture(n, dim, 16, 0.3, seed=seed)
    cent, ids = datasets.kmeans(base, K, iters=5, seed=seed + 1)
    # members off their centroids (a zero residual stalls fast_quantize,
    # inc/index/Quantizer.hpp:142-196)
    cent = cent + 0.01 * np.random.default_rng(seed + 2).standard_normal(cent.shape).astype(np.float32)
    return base, cent, ids.astype(np.uint32)


def _compare(ref_path, got_path):
    from erq_b200 import indexfile

    a = indexfile.read_index(ref_path)
    b = indexfile.read_index(got_path)
    assert (a.N, a.DIM, a.K, a.EX) == (b.N, b.DIM, b.K, b.EX)
    assert (a.sizes == b.sizes).all()
    for name in ("P", "centroids", "long_code", "xipnorm", "ids"):
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape, name
        bad = np.flatnonzero(x.reshape(-1).view(np.uint8) != y.reshape(-1).view(np.uint8))
        assert bad.size == 0, (name, bad[:10])
    D = a.D
    assert (a.short[:, :4 * D] == b.short[:, :4 * D]).all(), "1-bit codes"
    fa = a.short[:, 4 * D:].copy().view(np.float32)
    fb = b.short[:, 4 * D:].copy().view(np.float32)
    nb = (a.sizes.astype(np.int64) + 31) // 32
    used = np.zeros(fa.shape, bool)
    row = 0
    for s, m in zip(a.sizes.astype(np.int64), nb):
        for j in range(m):
            used[row + j, :min(32, s - 32 * j)] = True
        row += m
    assert (fa[used].view(np.uint32) == fb[used].view(np.uint32)).all(), "block factors"
    assert (fb[~used] == 0).all()


@pytest.mark.parametrize("bits", [3, 4, 5, 7, 8, 9])
def test_build_equals_create_index(tmp_path, bits):
    from erq_b200 import indexfile
    from erq_b200.build_index import build_index_gpu

    base, cent, ids = _case(2000, 100, 20, 30 + bits)
    ref_path = _reference_index(tmp_path, base, cent, ids, bits)
    P = indexfile.read_index(ref_path).P
    got = str(tmp_path / "gpu.index")
    build_index_gpu(base, cent, ids, bits, got, P=P)
    _compare(ref_path, got)


def test_build_equals_create_index_d1536(tmp_path):
    from erq_b200 import indexfile
    from erq_b200.build_index import build_index_gpu

    base, cent, ids = _case(3000, 1536, 24, 77, sphere=True)
    ref_path = _reference_index(tmp_path, base, cent, ids, 8)
    P = indexfile.read_index(ref_path).P
    got = str(tmp_path / "gpu1536.index")
    build_index_gpu(base, cent, ids, 8, got, P=P)
    _compare(ref_path, got)


def test_build_with_own_rotation_searches(tmp_path):
    """Without a given rotation the builder draws an orthogonal one; the index
    loads and its search equals the C restatement on it."""
    import oracle

    from erq_b200 import IVF, indexfile
    from erq_b200.build_index import build_index_gpu

    base, cent, ids = _case(3000, 128, 24, 5)
    path = str(tmp_path / "own.index")
    build_index_gpu(base, cent, ids, 5, path, seed=11)
    P = indexfile.read_index(path).P.astype(np.float64)
    assert np.abs(P @ P.T - np.eye(P.shape[0])).max() < 1e-5
    idx = IVF(path)
    q = idx.rotate(base[:16] + 0.01)
    oracle.build_oracle()
    o = oracle.Oracle(path)
    got_ids, got_d = idx.search_batch(q, 20, 6)
    want_ids, want_d = o.search(q, 20, 6)
    assert (got_ids == want_ids).all()
    assert (got_d.view(np.uint32) == want_d.view(np.uint32)).all()
    o.close()
    idx.free()


def test_create_index_driver_equals_reference(tmp_path):
    """extended-rabitq_b200/examples/erq_create_index.cpp - the reference's
    create_index over the C++ facade (IVF(n, dim, k, b) + construct + save)
    - reads the same files and, given the reference's rotation, writes the
    same index."""
    from conftest import PKG

    from erq_b200 import indexfile

    base, cent, ids = _case(2500, 200, 16, 91)
    ref_path = _reference_index(tmp_path, base, cent, ids, 7)
    P = indexfile.read_index(ref_path).P
    rot = tmp_path / "rotation.bin"
    P.astype(np.float32).tofile(rot)
    ref_copy = str(tmp_path / "ref.index")
    os.replace(ref_path, ref_copy)
    subprocess.run(["make", "-s", "-C", PKG, "bin/erq_create_index"], check=True)
    subprocess.run([os.path.join(PKG, "bin", "erq_create_index"), str(tmp_path / "data"), "bld",
                    "16", "7", str(rot)], check=True, stdout=subprocess.DEVNULL, timeout=300)
    _compare(ref_copy, ref_path)
