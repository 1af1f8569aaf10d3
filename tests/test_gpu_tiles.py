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


def test_window_push_at_scale_gives_the_same_bits(gpu):
    """The population-window push at scale: a 1.2M-neuron regional network (24 populations of
    ~50k neurons, in-degree 300, BF16) has ~4 windows per population, and a burst step hands each
    window dozens of 1024-row work units.  With the fixed-point push the window form (local:2016,
    its cross-population part on a second stream) and the register push must give the same bits:
    per-step counts, events, V and J after 600 steps."""
    spec = nw.structured_spec(1_200_000, 24, 300, seed=8)
    results = []
    for variant in [(E.PUSH_REG, 8), (E.PUSH_LOCAL, 2016)]:
        with E.Engine.structured(spec, weight_type=E.W_BF16, seed=77, ou=OU) as eng:
            eng.set_push_variant(*variant)
            if variant[0] == E.PUSH_LOCAL:
                assert eng.info().local_windows >= 48
            r = eng.run(600, syn_mode=E.SYN_PUSH_FIXED)
            results.append((r.freqs.copy(), r.events, eng.read_state(E.STATE_V), eng.read_state(E.STATE_J)))
    (f0, e0, v0, j0), (f1, e1, v1, j1) = results
    assert int((f0.sum(1) > spec.n // 100).sum()) >= 10, "the network must burst"
    assert np.array_equal(f0, f1) and e0 == e1
    assert np.array_equal(v0, v1) and np.array_equal(j0, j1)
