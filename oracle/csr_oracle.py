"""CPU oracle of CSR construction and of the regional-network edge stream --
TEST INFRASTRUCTURE ONLY (tests/, __graft_entry__.smoke(), bench.py's CPU leg).

* ``reference_out_csr`` restates the reference's out-degree CSR builder,
  ``parse_outdegree_from_numpy`` / ``parse_conn_table_from_numpy``
  (src/configuration.cpp:1079-1392, 1394-1667): synapses are stably sorted by
  (relative presynaptic block + block id, presynaptic neuron) -- thrust's
  ``stable_sort_by_key`` (configuration.cpp:227-249); rows are the presynaptic
  neurons with at least one synapse (``inner_conninds``), ``rowptr`` indexes them,
  and colind / weight / kind are permuted alike; the kind bit is
  ``input_channel_offset != 0`` (configuration.cpp:155-174, 1618, 1646).
* ``philox4x32_10`` restates the Philox4x32-10 generator of Salmon et al. (SC'11)
  in numpy, and ``structured_edges`` replays the engine's device edge stream
  (counter (post, k, 0x5EED0001, 0)) so small regional networks can be built on
  the host and compared with the device build bit for bit.
"""
from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
STREAM_EDGES = 0x5EED0001
MASK32 = np.uint64(0xFFFFFFFF)


def reference_out_csr(net, block_id=0):
    """Out-degree CSR of a block in the reference's layout.

    Returns dict(rows, row_ptr, post, kind, weight, perm).
    """
    pre = np.asarray(net["input_neuron_idx"], np.uint64)
    blk = np.asarray(net.get("input_block_idx", np.zeros(pre.shape[0], np.int16)), np.int64) + block_id
    key = (blk.astype(np.uint64) << np.uint64(32)) | pre
    perm = np.argsort(key, kind="stable")
    sk = key[perm]
    heads = np.ones(sk.shape[0], bool)
    heads[1:] = sk[1:] != sk[:-1]
    starts = np.nonzero(heads)[0]
    rows = (sk[starts] & MASK32).astype(np.uint32)
    row_ptr = np.concatenate([starts, [sk.shape[0]]]).astype(np.uint64)
    return dict(rows=rows, row_ptr=row_ptr,
                post=np.asarray(net["output_neuron_idx"], np.uint32)[perm],
                kind=(np.asarray(net["input_channel_offset"])[perm] != 0).astype(np.uint8),
                weight=np.asarray(net["weight"])[perm],
                perm=perm.astype(np.uint64))


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10 over uint32 arrays; returns four uint32 arrays."""
    c0, c1, c2, c3 = (np.asarray(c, np.uint64) for c in (c0, c1, c2, c3))
    k0, k1 = np.uint32(k0), np.uint32(k1)
    for _ in range(10):
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK32
        c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint64(k0), lo1, hi0 ^ c3 ^ np.uint64(k1), lo0
        k0 = np.uint32((int(k0) + int(W0)) & 0xFFFFFFFF)
        k1 = np.uint32((int(k1) + int(W1)) & 0xFFFFFFFF)
    return tuple(c.astype(np.uint32) for c in (c0, c1, c2, c3))


def structured_edges(spec):
    """Host replay of the device edge stream of a regional network spec.

    Returns the network in the reference's npz key set (post-major edges) plus
    the per-population property rows expanded to neurons.
    """
    n, k = spec.n, spec.in_degree
    off = spec.pop_offsets.astype(np.int64)
    post = np.repeat(np.arange(n, dtype=np.uint64), k)
    kk = np.tile(np.arange(k, dtype=np.uint64), n)
    a = np.repeat(np.repeat(np.arange(spec.n_pops), spec.pop_sizes), k)
    seed = int(spec.seed)
    x, y, z, w = philox4x32_10(post, kk, np.full(post.shape, STREAM_EDGES, np.uint64), np.zeros(post.shape, np.uint64),
                               seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    cdf = spec.src_cdf.astype(np.uint64)
    # first b with x < cdf[a, b]
    b = np.empty(post.shape[0], np.int64)
    for pa in range(spec.n_pops):
        m = a == pa
        b[m] = np.searchsorted(cdf[pa], x[m].astype(np.uint64), side="right")
    size = (off[b + 1] - off[b]).astype(np.uint64)
    same = b == a
    j = np.where(same,
                 off[b] + ((y.astype(np.uint64) * (size - np.uint64(1))) >> np.uint64(32)).astype(np.int64),
                 off[b] + ((y.astype(np.uint64) * size) >> np.uint64(32)).astype(np.int64))
    j = np.where(same & (j >= post.astype(np.int64)), j + 1, j)
    kind = ((j - off[b]) >= spec.pop_exc[b]).astype(np.uint8)
    if spec.dyadic_weights:
        w0 = (z >> np.uint32(24)).astype(np.float32) / np.float32(256.0)
        w1 = (w >> np.uint32(24)).astype(np.float32) / np.float32(256.0)
    else:
        w0 = (z >> np.uint32(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)
        w1 = (w >> np.uint32(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)
    return dict(property=spec.property_matrix(),
                input_block_idx=np.zeros(post.shape[0], np.int16),
                input_neuron_idx=j.astype(np.uint32),
                output_neuron_idx=post.astype(np.uint32),
                input_channel_offset=(kind * 2).astype(np.uint8),
                weight=np.stack([w0, w1], axis=1).astype(np.float32))
