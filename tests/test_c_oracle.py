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


def test_c_oracle64_equals_numpy_float64_oracle():
    """The FP64 restatement in C is bit-identical to LifOracle(dtype=float64)."""
    spec = nw.structured_spec(8000, 4, 300, seed=3)
    net = cc.structured_edges(spec)
    steps = 400
    z, _ = lo.torch_noise_stream(4, spec.n, steps, False)
    o64 = lo.LifOracle(net, dtype=np.float64)
    ref = np.array([o64.step(z[s].astype(np.float64))[0] for s in range(steps)])
    c = cc.COracle64(net)
    sp, counts, _, vt = c.run(z, n_v=16)
    assert ref[200:].mean() > 0.005
    assert np.array_equal(sp, ref)
    assert np.array_equal(counts, ref.sum(1))
    assert np.array_equal(c.V, o64.V) and np.array_equal(c.J, o64.J)
    assert np.array_equal(vt[-1], o64.V[:16].astype(np.float32))


def test_float32_clock_explains_the_rate_gap():
    """FP64 with only its clock rounded to float32 fires like the float32 model: the
    refractory test on block_new's float32 time is what moves the rate, not V."""
    spec = nw.structured_spec(30_000, 2, 1000, seed=1)
    net = cc.structured_edges(spec)
    steps, warm = 400, 150
    z = np.random.default_rng(7).standard_normal((steps, spec.n), dtype=np.float32)
    r64 = cc.COracle64(net).run(z)[0][warm:].mean()
    r64c = cc.COracle64(net).run(z, clock32=True)[0][warm:].mean()
    r32 = cc.COracle(net).run(z)[0][warm:].mean()
    assert abs(r64 - r32) > 0.05 * r32            # a visible gap on this network...
    assert abs(r64c - r32) < 0.002 * r32          # ...closed by the float32 clock alone
