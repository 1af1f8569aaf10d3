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


@pytest.mark.parametrize("prop_mode", [lo.PROP_THRESHOLD, lo.PROP_OR])
def test_event_driven_oracle_equals_full_sweep(prop_mode):
    """oracle_run_events (O(events) per step, threads over target ranges) gives the
    same float32 state as oracle_run (every in-edge each step): the double sums of
    weights that are multiples of 2^-24 are exact in any order."""
    spec = nw.structured_spec(12_000, 5, 300, seed=6)
    net = cc.structured_edges(spec)
    net["property"][:, 0] = 0.01
    steps = 300
    z, u = lo.torch_noise_stream(2, spec.n, steps, prop_mode != lo.PROP_THRESHOLD)
    a = cc.COracle(net, prop_mode=prop_mode)
    sp, counts, ev = a.run(z, u)
    pop = np.repeat(np.arange(spec.n_pops), spec.pop_sizes)
    b = cc.COracleEvents(net, pop, warm=0, prop_mode=prop_mode)
    _, counts_b, ev_b = b.run(z[:120], None if u is None else u[:120])
    _, counts_c, ev_c = b.run(z[120:], None if u is None else u[120:])
    assert counts.sum() > 0
    assert np.array_equal(np.concatenate([counts_b, counts_c]), counts) and ev_b + ev_c == ev
    for k in ("V", "J", "i_bg", "t_last", "I_syn"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    # running statistics equal the ones taken from the raster
    from tests.spike_stats import IsiMoments
    assert np.array_equal(b.pop_spikes, np.bincount(pop, weights=sp.sum(0), minlength=spec.n_pops).astype(np.int64))
    m = IsiMoments(spec.n, 0)
    m.add(sp[:77], 0)
    m.add(sp[77:], 77)
    assert m.count == int(b.isi[0]) and m.count > 0
    assert abs(m.cv() - b.isi_cv()) < 1e-12


def test_isi_moments_warm_up_and_chunks():
    rng = np.random.default_rng(3)
    r = rng.random((400, 50)) < 0.05
    warm = 100
    ref = []
    for j in range(50):
        t = np.nonzero(r[:, j])[0]
        t = t[t >= warm]
        ref.extend(np.diff(t))
    ref = np.asarray(ref, np.float64)
    from tests.spike_stats import IsiMoments
    m = IsiMoments(50, warm)
    for a in range(0, 400, 37):
        m.add(r[a:a + 37], a)
    assert m.count == ref.size
    assert abs(m.cv() - ref.std() / ref.mean()) < 1e-12
