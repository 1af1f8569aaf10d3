"""The C port of the oracle is bit-identical to the numpy oracle (which is pinned
to block_new), and its edge-stream replay equals the numpy replay."""
import numpy as np
import pytest

from dtb_b200 import network as nw
from oracle import c_oracle as cc
from oracle import csr_oracle as co
from oracle import lif_oracle as lo


@pytest.mark.parametrize("dyadic", [False, True])
@pytest.mark.parametrize("prop_mode", [lo.PROP_THRESHOLD, lo.PROP_NOISE, lo.PROP_OR])
def test_c_oracle_equals_numpy_oracle(dyadic, prop_mode):
    net = nw.make_uniform_block(3000, 60, seed=1, noise_rate=0.02, dyadic_weights=dyadic)
    steps = 250
    z, u = lo.torch_noise_stream(4, 3000, steps, prop_mode != lo.PROP_THRESHOLD)
    a = lo.LifOracle(net, prop_mode=prop_mode)
    ref = np.array([a.step(z[s], None if u is None else u[s])[0] for s in range(steps)])
    c = cc.COracle(net, prop_mode=prop_mode)
    sp, counts, _ = c.run(z, u)
    assert np.array_equal(sp, ref)
    assert np.array_equal(counts, ref.sum(1))
    assert np.array_equal(c.V, a.V)
    assert np.array_equal(c.J, a.J)
    assert np.array_equal(c.i_bg, a.i_bg)
    assert np.array_equal(c.t_last, a.t_last)


def test_c_edge_stream_equals_numpy_replay():
    spec = nw.structured_spec(5000, 7, 30, seed=13)
    a = co.structured_edges(spec)
    b = cc.structured_edges(spec)
    for k in ("input_neuron_idx", "output_neuron_idx", "input_channel_offset", "weight"):
        assert np.array_equal(a[k], b[k]), k


def test_c_oracle_structured_network_runs():
    spec = nw.structured_spec(20_000, 10, 200, seed=2)
    net = cc.structured_edges(spec)
    z, _ = lo.torch_noise_stream(0, spec.n, 50, False)
    c = cc.COracle(net)
    sp, counts, ev = c.run(z)
    assert sp.shape == (50, spec.n) and counts.sum() == sp.sum()
