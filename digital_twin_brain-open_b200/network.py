"""Synthetic Digital-Twin-Brain networks: host-side specs and the small generators.

Two kinds of network are built here.

* ``make_uniform_block`` -- the plain LIF block the reference runs on its CPU
  model (``models/block_new.py``): N neurons in ONE population, the first 80 %
  excitatory, fixed in-degree K with presynaptic sources drawn uniformly without
  replacement and without self-loops (``numpy.random.default_rng(seed)``), weight
  pairs ~U(0,1) float32.  It is returned in the reference's on-disk key set
  (``src/configuration.cpp:1094-1098, 1508-1517, 1789``): ``property [N,22] f32``,
  ``input_block_idx [S] i16`` (relative block id, 0 = this block),
  ``input_neuron_idx [S] u32``, ``output_neuron_idx [S] u32``,
  ``input_channel_offset [S] u8`` (0 = AMPA/NMDA pair, 2 = GABAa/GABAb pair, as
  written by ``python/make_block.py:305-310``) and ``weight [S,2]``.  Edges are
  post-major, the order ``make_block.py`` writes.

* ``StructuredSpec`` -- the regional networks (millions of neurons, hundreds of
  populations, distance-dependent population coupling).  Only the per-population
  tables live on the host; the edges themselves are generated on the GPU by a
  counter-based Philox stream (``dtb_create_structured`` in the C-ABI), edge
  ``(post, k)`` from counter ``(post, k, STREAM_EDGES, 0)``, so any edge can be
  regenerated independently and the device build is reproducible bit for bit.

The 22 property columns follow ``python/make_block.py:426-464``:
0 noise_rate, 1 blocked_in_stat, 2 I_ext, 3 population id, 4 C, 5 T_ref, 6 g_L,
7 V_L, 8 V_th, 9 V_reset, 10-13 g_ui, 14-17 V_ui, 18-21 tau_ui.
"""
from __future__ import annotations

import dataclasses
import hashlib

import numpy as np

# LIF / OU parameters shared by every synthetic configuration.
LIF_PARAMS = dict(C=1.0, g_L=0.03, V_L=-75.0, V_th=-50.0, V_reset=-65.0, T_ref=5.0,
                  g_ui=(0.01, 0.002, 0.04, 0.002), V_ui=(0.0, 0.0, -70.0, -100.0),
                  tau_ui=(2.0, 40.0, 10.0, 50.0))
OU_PARAMS = dict(mean=0.6, sigma=0.2, tau=10.0)
DT_MS = 0.1

# Philox stream ids (the third counter word) used by the device generator.
STREAM_EDGES = 0x5EED0001

# Weight encodings understood by the engine (``dtb_weight_type`` in the C-ABI).
WEIGHT_F32 = 0
WEIGHT_BF16 = 1
WEIGHT_F16 = 2
WEIGHT_U8 = 3   # uint8 / 255, the reference's "int8" directory type
WEIGHT_F64 = 4


def lif_property(n, pop_ids, noise_rate=0.0, i_ext=0.0, g_ui=None):
    """Property matrix ``[n, 22]`` float32 with the shared LIF parameters.

    ``g_ui`` may be ``[n, 4]`` to override the receptor conductances per neuron.
    """
    p = np.zeros((n, 22), np.float32)
    p[:, 0] = noise_rate
    p[:, 1] = 0.0
    p[:, 2] = i_ext
    p[:, 3] = pop_ids
    p[:, 4] = LIF_PARAMS["C"]
    p[:, 5] = LIF_PARAMS["T_ref"]
    p[:, 6] = LIF_PARAMS["g_L"]
    p[:, 7] = LIF_PARAMS["V_L"]
    p[:, 8] = LIF_PARAMS["V_th"]
    p[:, 9] = LIF_PARAMS["V_reset"]
    p[:, 10:14] = LIF_PARAMS["g_ui"] if g_ui is None else g_ui
    p[:, 14:18] = LIF_PARAMS["V_ui"]
    p[:, 18:22] = LIF_PARAMS["tau_ui"]
    return p


def make_uniform_block(n=10_000, k=100, exc_frac=0.8, seed=0, noise_rate=0.0,
                       dyadic_weights=False):
    """The plain block: one population, fixed in-degree, uniform sources.

    ``dyadic_weights`` quantises every weight to a multiple of 1/256, which makes
    every sum of up to 2**15 weights exact in float32 whatever the summation
    order; parity tests use it to compare GPU and oracle bit for bit.
    """
    rng = np.random.default_rng(seed)
    n_exc = int(round(n * exc_frac))
    pre = np.empty(n * k, np.uint32)
    for i in range(n):
        c = rng.choice(n - 1, k, replace=False)
        c[c >= i] += 1
        pre[i * k:(i + 1) * k] = c
    post = np.repeat(np.arange(n, dtype=np.uint32), k)
    w = rng.random((n * k, 2), dtype=np.float32)
    if dyadic_weights:
        w = (np.floor(w * 256.0) / 256.0).astype(np.float32)
    kind = np.where(pre >= n_exc, 2, 0).astype(np.uint8)
    return dict(
        property=lif_property(n, 0, noise_rate=noise_rate),
        input_block_idx=np.zeros(n * k, np.int16),
        input_neuron_idx=pre,
        output_neuron_idx=post,
        input_channel_offset=kind,
        weight=w,
    )


def arrays_digest(arrays):
    """sha256 over the network arrays, to pin a regenerated network to a fixture."""
    h = hashlib.sha256()
    for key in ("property", "input_block_idx", "input_neuron_idx", "output_neuron_idx",
                "input_channel_offset", "weight"):
        a = np.ascontiguousarray(arrays[key])
        h.update(key.encode())
        h.update(str(a.dtype).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def write_npz(path, arrays):
    """Write a block in the reference's npz key set (``np.savez``, uncompressed)."""
    np.savez(path, **{k: arrays[k] for k in ("property", "input_block_idx", "input_neuron_idx",
                                             "output_neuron_idx", "input_channel_offset", "weight")})


@dataclasses.dataclass
class StructuredSpec:
    """Per-population tables of a regional network; edges are generated on device.

    * ``pop_sizes[P]``: neurons per population, contiguous, in id order;
    * ``pop_exc[P]``: the first ``pop_exc[b]`` neurons of population b are excitatory;
    * ``src_cdf[P, P]`` (u64): row a is the cumulative distribution of the source
      population of an edge into population a, scaled to 2**32 (last entry == 2**32);
      the source population of edge (post, k) is the first b with r0 < src_cdf[a, b];
    * ``in_degree``: edges per post neuron;
    * ``g_ui[P, 4]``: receptor conductances per population.
    """
    pop_sizes: np.ndarray
    pop_exc: np.ndarray
    src_cdf: np.ndarray
    in_degree: int
    seed: int
    g_ui: np.ndarray
    dyadic_weights: bool = False

    @property
    def n(self):
        return int(self.pop_sizes.sum())

    @property
    def n_pops(self):
        return int(self.pop_sizes.shape[0])

    @property
    def pop_offsets(self):
        return np.concatenate([[0], np.cumsum(self.pop_sizes)]).astype(np.int64)

    @property
    def n_edges(self):
        return self.n * self.in_degree

    def property_rows(self, pop_id_base=0):
        """One property row per population, ``[P, 22]`` (column 3 = population id)."""
        return lif_property(self.n_pops, np.arange(self.n_pops) + pop_id_base, g_ui=self.g_ui)

    def property_matrix(self, pop_id_base=0):
        pops = np.repeat(np.arange(self.n_pops), self.pop_sizes) + pop_id_base
        g = np.repeat(self.g_ui, self.pop_sizes, axis=0)
        return lif_property(self.n, pops, g_ui=g)


def split_sizes(n, weights):
    """Integer sizes proportional to ``weights`` summing to n (largest remainder)."""
    raw = np.asarray(weights, np.float64) / np.sum(weights) * n
    base = np.floor(raw).astype(np.int64)
    rem = n - int(base.sum())
    order = np.argsort(-(raw - base), kind="stable")
    base[order[:rem]] += 1
    return base


def structured_spec(n, n_pops, in_degree, seed, self_frac=0.7, length=20.0, box=100.0,
                    exc_frac=0.8, g_scale=None, dyadic_weights=False, min_pop=8):
    """Regional network construction (5M-neuron regional network and its relatives).

    Population sizes ~ lognormal(0, 0.5) normalised to n (largest remainder, each at
    least ``min_pop``); coordinates ~U[0, box]^3; P_aa = self_frac and
    P_ab = (1 - self_frac) exp(-d_ab / length) / sum_{c != a} exp(-d_ac / length).
    ``g_scale[P, 4]`` multiplies the base receptor conductances per population.
    """
    rng = np.random.default_rng(seed)
    w = rng.lognormal(0.0, 0.5, n_pops)
    sizes = split_sizes(n - min_pop * n_pops, w) + min_pop
    xyz = rng.uniform(0.0, box, (n_pops, 3))
    d = np.sqrt(((xyz[:, None, :] - xyz[None, :, :]) ** 2).sum(-1))
    off = np.exp(-d / length)
    np.fill_diagonal(off, 0.0)
    if n_pops > 1:
        prob = (1.0 - self_frac) * off / off.sum(1, keepdims=True)
        np.fill_diagonal(prob, self_frac)
    else:
        prob = np.ones((1, 1))
    cdf = np.cumsum(prob, axis=1)
    cdf = cdf / cdf[:, -1:]
    src_cdf = np.minimum(np.round(cdf * 2.0 ** 32), 2.0 ** 32).astype(np.uint64)
    src_cdf[:, -1] = np.uint64(2 ** 32)
    exc = np.round(sizes * exc_frac).astype(np.int64)
    base = np.asarray(LIF_PARAMS["g_ui"], np.float32)
    g = np.tile(base, (n_pops, 1)).astype(np.float32)
    if g_scale is not None:
        g = (g * np.asarray(g_scale, np.float32)).astype(np.float32)
    return StructuredSpec(pop_sizes=sizes.astype(np.int64), pop_exc=exc, src_cdf=src_cdf,
                          in_degree=int(in_degree), seed=int(seed), g_ui=g,
                          dyadic_weights=dyadic_weights)


def regional_5m_spec(seed=1, n=5_000_000, n_pops=200, in_degree=1000):
    """The 5M-neuron, 200-population, in-degree-1000 regional network."""
    return structured_spec(n, n_pops, in_degree, seed)


def ensemble_specs(n_members=64, seed=3, n_lo=20_000, n_hi=400_000,
                   degrees=(100, 200, 500), pops_lo=10, pops_hi=50):
    """Data-assimilation ensemble members: uneven sizes, degrees and population counts.

    Each member draws its own g_ui per population from U(0.5, 1.5) x base.
    """
    rng = np.random.default_rng(seed)
    specs = []
    for m in range(n_members):
        n = int(rng.integers(n_lo, n_hi + 1))
        k = int(rng.choice(degrees))
        p = int(rng.integers(pops_lo, pops_hi + 1))
        scale = rng.uniform(0.5, 1.5, (p, 4))
        specs.append(structured_spec(n, p, k, seed * 1000 + m + 1, g_scale=scale))
    return specs
