"""Blocks on disk in every weight type, and the Gamma resampling of properties.

* The reference reads ``block_<i>.npz`` with its weight type taken from the directory
  in the path -- "/single", "/half", "/int8" or "/uint8", "/double"
  (src/configuration.cpp:1411-1435) -- and decodes float16 as is, uint8 as value /
  255 and float64 narrowed to float32 (src/stage/presynaptic_voltage.cpp:153-176).
  Loaded through ``dtb_create_from_npz`` each block runs exactly like the oracle fed
  the decoded float32 weights (exact push: bit for bit).
* ``dtb_update_gamma`` (Updategamma, src/stage/property.cpp:494-651) draws every
  neuron's property of the addressed population from Gamma(alpha, 1) / beta: the
  draws have mean alpha / beta and variance alpha / beta^2, and nothing else changes.
"""
import os

import numpy as np
import pytest

from dtb_b200 import engine as E
from dtb_b200 import network as nw
from oracle import c_oracle as cc
from oracle import lif_oracle as lo

pytestmark = pytest.mark.gpu

CASES = [("single", np.float32, E.W_F32), ("half", np.float16, E.W_F16), ("uint8", np.uint8, E.W_U8),
         ("int8", np.uint8, E.W_U8), ("double", np.float64, E.W_F32)]


def _encode(w, dtype):
    """File weights of `dtype` and the float32 values the reference decodes from them."""
    if dtype == np.uint8:
        u = np.round(w * 255.0).astype(np.uint8)
        return u, u.astype(np.float32) / np.float32(255.0)
    if dtype == np.float16:
        h = w.astype(np.float16)
        return h, h.astype(np.float32)
    return w.astype(dtype), w.astype(np.float32)


@pytest.mark.parametrize("directory,dtype,device_type", CASES, ids=[c[0] for c in CASES])
def test_block_files_in_every_weight_type(gpu, tmp_path, directory, dtype, device_type):
    net = nw.make_uniform_block(4000, 100, seed=6)
    stored, decoded = _encode(net["weight"], dtype)
    d = tmp_path / "net" / directory
    os.makedirs(d)
    nw.write_npz(str(d / "block_0.npz"), dict(net, weight=stored))
    ref_net = dict(net, weight=decoded)
    steps = 400
    z, _ = lo.torch_noise_stream(3, 4000, steps, False)
    ref = cc.COracle(ref_net)
    sp, _, _ = ref.run(z)
    with E.Engine.from_npz(str(d / "block_0.npz"), weight_type=device_type, seed=1) as eng:
        assert eng.info().weight_type == device_type
        _, _, _, _, w = eng.read_out_csr()
        assert np.array_equal(np.sort(w[:, 0]), np.sort(decoded[:, 0]))
        eng.set_noise_injected(z)
        r = eng.run(steps, record_spikes=True, syn_mode=E.SYN_PUSH_EXACT)
        assert sp[200:].mean() > 0.002
        assert np.array_equal(r.spikes, sp)
        assert np.array_equal(eng.read_state(E.STATE_V), ref.V)
        assert np.array_equal(eng.read_state(E.STATE_J), ref.J.T)


@pytest.mark.parametrize("alpha,beta", [(4.0, 2000.0), (0.5, 50.0)])
def test_gamma_draws(gpu, alpha, beta):
    """About 1.1M draws: the sample mean's relative spread is 1 / sqrt(alpha n) (0.14 % at
    alpha = 0.5) and the sample variance's sqrt((2 + 6 / alpha) / n) (0.36 %), so the 1 %
    and 3 % bars sit beyond six standard deviations for both shapes."""
    spec = nw.structured_spec(1_300_000, 2, 5, seed=3)
    g = E.PROP_IDS["CONDUCT_G_AMPA"]
    with E.Engine.structured(spec) as eng:
        before = {p: eng.read_property(p) for p in range(20)}
        eng.update_gamma([g], [0], [alpha], [beta])                     # population 0: 1,181,350 neurons
        after = {p: eng.read_property(p) for p in range(20)}
        lo_, hi_ = spec.pop_offsets[0], spec.pop_offsets[1]
        x = after[g][lo_:hi_].astype(np.float64)
        assert x.size > 1_000_000
        assert abs(x.mean() / (alpha / beta) - 1.0) < 0.01
        assert abs(x.var() / (alpha / beta ** 2) - 1.0) < 0.03
        assert np.array_equal(after[g][hi_:], before[g][hi_:])          # other population untouched
        for p in range(20):
            if p != g:
                assert np.array_equal(after[p], before[p]), p            # other properties untouched
        # a second call draws new values; the network runs on them
        eng.update_gamma([g], [0], [alpha], [beta])
        assert not np.array_equal(eng.read_property(g)[lo_:hi_], after[g][lo_:hi_])
        assert eng.run(50).freqs.shape == (50, 2)
