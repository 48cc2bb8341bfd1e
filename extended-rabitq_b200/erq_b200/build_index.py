"""Index construction on a GPU with torch, writing the reference's index file.

Follows DataQuantizer::quantize (inc/index/Quantizer.hpp:233-311) for each
cluster: rotate the padded data and centroid, take the residual, its sign
bits (the 1-bit FastScan code) and its normalised magnitude, quantise the
magnitude to EX bits, flip the code on negative dimensions, and store
||o - c|| as the block factor (HIGH_ACC_FAST_SCAN).  Used to make the large
benchmark indexes quickly; the small parity fixtures come from the
reference's own create_index.

Differences from the reference's builder, none of which touch the search:
* the rotation is any orthogonal matrix (the reference draws its own);
* the EX-bit rescaling factor t is found by a two-level grid search over
  [t_start, t_end) instead of the exact critical-point sweep of
  fast_quantize (inc/index/Quantizer.hpp:138-219), in float32, so a few codes
  may differ by one level; the factor xipnorm is computed from the code that
  is stored, so the distance estimate stays consistent;
* padding lanes of the last block of a cluster carry factor 0 (the
  reference leaves them uninitialised; the search never reads them).
"""
from __future__ import annotations

import numpy as np

from .indexfile import IndexArrays

PERM0 = [0, 8, 1, 9, 2, 10, 3, 11, 4, 12, 5, 13, 6, 14, 7, 15]


def random_rotation(D: int, seed: int = 0):
    """An orthogonal D x D matrix P (rows of Q^T from a float64 QR)."""
    import torch

    g = torch.Generator().manual_seed(seed)
    a = torch.randn(D, D, generator=g, dtype=torch.float64)
    q, r = torch.linalg.qr(a)
    q = q * torch.sign(torch.diagonal(r))[None, :]
    return q.T.contiguous().float()


def _ex_codes(o, ex_bits: int, grid: int = 64):
    """Grid search of fast_quantize's rescaling factor for each row of
    o = |normalised residual| (float32 [n, D]); returns (codes uint8, ip_norm)."""
    import torch

    B = (1 << ex_bits) - 1
    max_o = o.max(1).values.clamp_min(1e-30)
    t_start = (B // 3) / max_o
    t_end = (B + 10) / max_o
    lin = torch.linspace(0.0, 1.0, grid, device=o.device)

    def score(ts):
        ob = torch.floor(ts[:, :, None] * o[:, None, :] + 1e-5).clamp_(max=B)
        ob += 0.5
        num = (ob * o[:, None, :]).sum(2)
        den = (ob * ob).sum(2)
        return num / den.sqrt()

    ts = t_start[:, None] + (t_end - t_start)[:, None] * lin[None, :]
    best = score(ts).argmax(1)
    t0 = ts.gather(1, best[:, None])[:, 0]
    step = (t_end - t_start) / (grid - 1)
    ts2 = (t0 - step)[:, None] + (2 * step)[:, None] * lin[None, :]
    ts2 = torch.maximum(ts2, t_start[:, None])
    best2 = score(ts2).argmax(1)
    t = ts2.gather(1, best2[:, None])[:, 0]
    code = torch.floor(t[:, None] * o + 1e-5).clamp_(max=B)
    numerator = ((code.double() + 0.5) * o.double()).sum(1)
    ip_norm = (1.0 / numerator).float()
    ip_norm = torch.where(torch.isfinite(ip_norm), ip_norm, torch.ones_like(ip_norm))
    return code.to(torch.uint8), ip_norm


def pack_ex_codes(v, ex_bits: int):
    """store_compacted_code (inc/index/Quantizer.hpp:491-631) for rows of
    D byte values v (uint8 [n, D]) -> uint8 [n, D*EX/8]."""
    import torch

    n, D = v.shape
    v = v.to(torch.int32)
    if ex_bits == 8:
        return v.to(torch.uint8)
    if ex_bits == 4:
        x = v.view(n, D // 32, 2, 16)
        return (x[:, :, 0] | (x[:, :, 1] << 4)).to(torch.uint8).reshape(n, D // 2)
    g = v.view(n, D // 64, 4, 16)  # [n, group, sub, lane]: dim 16*sub + lane
    if ex_bits in (2, 3):
        low = g & 3
        body = (low[:, :, 0] | (low[:, :, 1] << 2) | (low[:, :, 2] << 4) | (low[:, :, 3] << 6))
        if ex_bits == 2:
            return body.to(torch.uint8).reshape(n, D // 4)
        top = _top_bits(v.view(n, D // 64, 64), 2)
        return torch.cat([body, top], 2).to(torch.uint8).reshape(n, D * 3 // 8)
    # 6 or 7
    low = g & 63
    b0 = low[:, :, 0] | ((low[:, :, 2] << 2) & 0xC0)
    b1 = low[:, :, 1] | ((low[:, :, 3] << 2) & 0xC0)
    b2 = (low[:, :, 2] & 15) | ((low[:, :, 3] & 15) << 4)
    body = torch.cat([b0, b1, b2], 2)
    if ex_bits == 6:
        return body.to(torch.uint8).reshape(n, D * 6 // 8)
    top = _top_bits(v.view(n, D // 64, 64), 6)
    return torch.cat([body, top], 2).to(torch.uint8).reshape(n, D * 7 // 8)


def _top_bits(v64, bit: int):
    """8 bytes per 64 dims: bit j of byte m is bit `bit` of dim 8j + m."""
    import torch

    b = (v64 >> bit) & 1                      # [n, G, 64]
    b = b.view(*b.shape[:2], 8, 8)            # [n, G, j, m] = dim 8j + m
    w = (1 << torch.arange(8, device=v64.device, dtype=torch.int32))[None, None, :, None]
    return (b * w).sum(2)                     # [n, G, m]


def build_index_torch(base, centroids, cluster_ids, bits: int, P=None, seed: int = 0,
                      chunk: int = 1024) -> IndexArrays:
    """Quantise ``base`` [N, DIM] (torch float32, any device) into an
    IndexArrays of the reference format.  ``cluster_ids`` [N] in [0, K)."""
    import torch

    dev = base.device
    N, DIM = base.shape
    K = centroids.shape[0]
    EX = bits - 1
    if EX not in (2, 3, 4, 6, 7, 8):
        raise ValueError(f"bits={bits}: total bits must be 3,4,5,7,8 or 9")
    D = (DIM + 63) // 64 * 64
    P = (random_rotation(D, seed) if P is None else torch.as_tensor(P, dtype=torch.float32))
    P = P.to(dev)
    cluster_ids = cluster_ids.to(dev).long()
    order = torch.argsort(cluster_ids, stable=True)
    sizes = torch.bincount(cluster_ids, minlength=K)
    nblocks = (sizes + 31) // 32
    first_block = torch.cumsum(nblocks, 0) - nblocks
    first_vec = torch.cumsum(sizes, 0) - sizes
    total_blocks = int(nblocks.sum())

    prev_tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        cpad = torch.zeros(K, D, device=dev)
        cpad[:, :DIM] = centroids.to(dev).float()
        CP = cpad @ P
        nib = torch.zeros(N, D // 4, dtype=torch.uint8, device=dev)
        onorm = torch.zeros(N, device=dev)
        long_code = torch.empty(N, D * EX // 8, dtype=torch.uint8, device=dev)
        xip = torch.empty(N, device=dev)
        for s in range(0, N, chunk):
            idx = order[s:s + chunk]
            c = cluster_ids[idx]
            x = torch.zeros(idx.numel(), D, device=dev)
            x[:, :DIM] = base[idx].float()
            xp = x @ P - CP[c]
            pos = xp > 0
            nrm = xp.norm(dim=1, keepdim=True)
            xn = torch.where(nrm > 0, xp / nrm.clamp_min(1e-30), xp)
            dist2c = (base[idx].float() - centroids.to(dev)[c].float()).pow(2).sum(1).sqrt()
            code, ip_norm = _ex_codes(xn.abs(), EX)
            mask = (1 << EX) - 1
            code = torch.where(pos, code, (~code) & mask)
            long_code[s:s + idx.numel()] = pack_ex_codes(code, EX)
            xip[s:s + idx.numel()] = ip_norm * 2 * dist2c
            onorm[s:s + idx.numel()] = dist2c
            b = pos.view(-1, D // 4, 4).to(torch.uint8)
            nib[s:s + idx.numel()] = (b[:, :, 0] << 3) | (b[:, :, 1] << 2) | (b[:, :, 2] << 1) | b[:, :, 3]
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev_tf32

    # FastScan blocks (pack_codes, inc/index/fastscan/pack_codes.hpp:33-98)
    sorted_c = cluster_ids[order]
    rank = torch.arange(N, device=dev) - first_vec[sorted_c]
    blk = first_block[sorted_c] + rank // 32
    lane = rank % 32
    lanes = torch.zeros(total_blocks, 32, D // 4, dtype=torch.uint8, device=dev)
    lanes[blk, lane] = nib
    fac = torch.zeros(total_blocks, 32, device=dev)
    fac[blk, lane] = onorm
    perm = torch.tensor(PERM0, device=dev)
    lo = lanes[:, perm, :]          # [blocks, 16 (byte j), groups]
    hi = lanes[:, perm + 16, :]
    codes = (lo | (hi << 4)).permute(0, 2, 1).contiguous().view(total_blocks, 4 * D)
    short = torch.cat([codes, fac.view(torch.uint8).view(total_blocks, 128)], 1)

    return IndexArrays(
        N=N, DIM=DIM, K=K, EX=EX,
        sizes=sizes.cpu().numpy().astype(np.uint64),
        P=P.cpu().numpy(),
        centroids=CP.cpu().numpy(),
        short=short.cpu().numpy(),
        long_code=long_code.cpu().numpy(),
        xipnorm=xip.cpu().numpy(),
        ids=order.cpu().numpy().astype(np.uint32),
    )


def build_index_gpu(base, centroids, cluster_ids, bits: int, path, P=None, seed: int = 0,
                    device: int = 0) -> None:
    """IVF(n, dim, k, bits) + construct + save on the GPU (erq_build_index):
    the reference's index bytes for the same data, centroids, cluster ids and
    rotation P (drawn from ``seed`` when None).  Arrays: numpy or torch."""
    import ctypes as C
    import os

    from ._lib import check, load_library

    def ptr(a):
        return None if a is None else C.c_void_p(
            a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data)

    if not hasattr(base, "data_ptr"):
        base = np.ascontiguousarray(base, np.float32)
    if not hasattr(centroids, "data_ptr"):
        centroids = np.ascontiguousarray(centroids, np.float32)
    if not hasattr(cluster_ids, "data_ptr"):
        cluster_ids = np.ascontiguousarray(cluster_ids, np.uint32)
    if P is not None and not hasattr(P, "data_ptr"):
        P = np.ascontiguousarray(P, np.float32)
    n, dim = base.shape
    check(load_library().erq_build_index(ptr(base), n, dim, ptr(centroids), centroids.shape[0],
                                         ptr(cluster_ids), bits, ptr(P), seed,
                                         os.fsencode(os.fspath(path)), device))
