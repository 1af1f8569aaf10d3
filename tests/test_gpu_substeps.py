"""Substeps (RunRequest.t_steps > 1): each step runs t_steps substeps of dt / t_steps
-- OU, membrane update and threshold, receptor decay with no input between them --
with the spikes OR-ed over the substeps and propagated once after the last
(tools/dist_simulator.cpp:2085-2112, src/block.cpp:729-737, 875-888), checked
against the oracle's restatement of that loop (LifOracle.step_substeps).

Exact and fixed-point push sum the input exactly for these weights, so spikes,
counts, V, J, the OU current and t_last equal the oracle bit for bit; the float
push equals it until the first threshold divergence, V within 1e-5 before it.
"""
import numpy as np
import pytest

from dtb_b200 import engine as E
from dtb_b200 import network as nw
from oracle import lif_oracle as lo

pytestmark = pytest.mark.gpu

V_RTOL = 1e-5


OU = (0.7, 0.2, 10.0)     # OU mean 0.7: the 3000-neuron block fires from step ~50 with substeps


def _oracle(net, z, steps, ts):
    dts = float(np.float32(0.1) / np.float32(ts))
    o = lo.LifOracle(net, dt=dts, ou=OU)
    rec = np.array([o.step_substeps(z[ts * s:ts * (s + 1)]) for s in range(steps)])
    return o, rec


@pytest.mark.parametrize("ts", [2, 3, 5])
@pytest.mark.parametrize("syn", [E.SYN_PUSH_EXACT, E.SYN_PUSH_FIXED], ids=["exact", "fixed"])
def test_substeps_bit_exact(gpu, syn, ts):
    net = nw.make_uniform_block(3000, 100, seed=2)
    steps = 300
    z, _ = lo.torch_noise_stream(7, 3000, steps * ts, False)
    o, rec = _oracle(net, z, steps, ts)
    with E.Engine.from_arrays(net, seed=1, ou=OU) as eng:
        eng.set_noise_injected(z)
        eng.set_samples(np.arange(0, 3000, 97))
        r = eng.run(steps, record_spikes=True, vmean=True, sample_spike=True, sample_v=True, syn_mode=syn,
                    t_steps=ts)
        assert rec[steps // 2:].mean() > 0.002
        assert np.array_equal(r.spikes, rec)
        assert np.array_equal(r.freqs[:, 0], rec.sum(1))
        assert np.array_equal(r.sample_spike.astype(bool), rec[:, ::97])
        assert np.array_equal(eng.read_state(E.STATE_V), o.V)
        assert np.array_equal(eng.read_state(E.STATE_J), o.J.T)
        assert np.array_equal(eng.read_state(E.STATE_I_OU), o.i_bg)
        assert np.array_equal(eng.read_state(E.STATE_T_LAST), o.t_last)
        assert np.array_equal(r.sample_v[-1], o.V[::97])
        inf = eng.info()
        assert inf.step == steps and inf.t == o.t     # the clock advanced by dt / ts per substep


def test_substeps_float_push_until_divergence(gpu):
    net = nw.make_uniform_block(3000, 100, seed=2)
    steps, ts = 300, 2
    z, _ = lo.torch_noise_stream(8, 3000, steps * ts, False)
    o = lo.LifOracle(net, dt=float(np.float32(0.1) / np.float32(ts)), ou=OU)
    vs, rec = [], []
    for s in range(steps):
        rec.append(o.step_substeps(z[ts * s:ts * (s + 1)]))
        vs.append(o.V[:64].copy())
    rec = np.array(rec)
    with E.Engine.from_arrays(net, seed=1, ou=OU) as eng:
        eng.set_noise_injected(z)
        eng.set_samples(np.arange(64))
        r = eng.run(steps, record_spikes=True, sample_v=True, syn_mode=E.SYN_PUSH, t_steps=ts)
    bad = np.nonzero((r.spikes != rec).any(axis=1))[0]
    upto = int(bad[0]) if bad.size else steps
    assert upto > 20 and rec[:upto].sum() > 0
    assert np.allclose(r.sample_v[:upto], np.array(vs)[:upto], rtol=V_RTOL, atol=0)


def test_substeps_continue_across_runs_and_chunks(gpu):
    """Two runs of t_steps = 3 give the same bits as one, and a plain run in between
    leaves the substep constants behind (the view returns to dt)."""
    spec = nw.structured_spec(20_000, 6, 200, seed=3)
    with E.Engine.structured(spec, seed=5) as a, E.Engine.structured(spec, seed=5) as b:
        fa = np.concatenate([a.run(150, syn_mode=E.SYN_PUSH_FIXED, t_steps=3).freqs,
                             a.run(250, syn_mode=E.SYN_PUSH_FIXED, t_steps=3).freqs])
        fb = b.run(400, syn_mode=E.SYN_PUSH_FIXED, t_steps=3).freqs
        assert np.array_equal(fa, fb) and fa.sum() > 0
        assert np.array_equal(a.read_state(E.STATE_V), b.read_state(E.STATE_V))
        ra = a.run(50, syn_mode=E.SYN_PUSH_FIXED)
        rb = b.run(50, syn_mode=E.SYN_PUSH_FIXED)
        assert np.array_equal(ra.freqs, rb.freqs)
        assert abs(a.info().t - (400 * 3 * np.float32(0.1 / 3) + 50 * 0.1)) < 1e-2


def test_substep_requests_are_validated(gpu):
    net = nw.make_uniform_block(1000, 20, seed=1)
    with E.Engine.from_arrays(net, pull=True) as eng:
        with pytest.raises(E.DtbError) as ei:
            eng.run(10, use_ou=False, t_steps=2)          # the reference answers SNN_INVALID_PARAMETER
        assert ei.value.status == E.INVALID_PARAMETER
        with pytest.raises(E.DtbError) as ei:
            eng.run(10, syn_mode=E.SYN_PULL, t_steps=2)
        assert ei.value.status == E.UNSUPPORTED
        with pytest.raises(E.DtbError) as ei:
            eng.run(10, t_steps=300)
        assert ei.value.status == E.INVALID_PARAMETER
        r1 = eng.run(20, t_steps=1, syn_mode=E.SYN_PUSH_EXACT)
        assert r1.freqs.shape == (20, 1)
