"""One network larger than the LIF kernel's persistent grid: 1,000,000 neurons are
977 tiles of 1024 for 444 CTAs (3 per SM on 148 SMs), so every CTA steps two or
three tiles in a row -- the second tile's copies in flight in the bulk-copy ring
while the first is stepped, the statistics slots alternating by tile parity, one
CTA barrier per tile.  Smaller networks give each CTA one tile and never reach
that path.  A strong OU drive (mean 3) makes the whole network fire in bursts of
~5 % of the neurons per step; exact and fixed-point push must equal the oracle
bit for bit (models/block_new.py:122-158): spikes, per-step counts, events, V, J.
"""
import numpy as np
import pytest

from dtb_b200 import engine as E
from dtb_b200 import network as nw
from oracle import c_oracle as cc
from oracle import lif_oracle as lo

pytestmark = pytest.mark.gpu

N, K, STEPS, CHUNK = 1_000_000, 20, 180, 60
OU = (3.0, 0.2, 10.0)


@pytest.fixture(scope="module")
def block1m():
    return nw.make_uniform_block(N, K, seed=3)


@pytest.mark.parametrize("syn", [E.SYN_PUSH_EXACT, E.SYN_PUSH_FIXED], ids=["exact", "fixed"])
def test_consecutive_tiles_per_cta_bit_exact(gpu, block1m, syn):
    ref = cc.COracle(block1m, ou=OU)
    spiking_steps = 0
    with E.Engine.from_arrays(block1m, seed=1, ou=OU) as eng:
        if syn == E.SYN_PUSH_FIXED:
            assert eng.info().fixed_shift > 0
        for z, _ in lo.torch_noise_chunks(7, N, STEPS, CHUNK):
            sp, counts, ev = ref.run(z)
            eng.set_noise_injected(z)
            r = eng.run(z.shape[0], record_spikes=True, syn_mode=syn)
            assert np.array_equal(r.spikes, sp)
            assert np.array_equal(r.freqs[:, 0], counts)
            assert r.events == ev
            spiking_steps += int((counts > N // 100).sum())
        assert np.array_equal(eng.read_state(E.STATE_V), ref.V)
        assert np.array_equal(eng.read_state(E.STATE_J), ref.J.T)
        assert np.array_equal(eng.read_state(E.STATE_I_OU), ref.i_bg)
    assert spiking_steps >= 10, "the network must burst"
