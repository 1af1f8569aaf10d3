"""Batched form: members advanced together give exactly their solo results."""
import numpy as np
import pytest

from dtb_b200 import engine as E
from dtb_b200 import network as nw
from oracle import lif_oracle as lo

pytestmark = pytest.mark.gpu

SPECS = [(12_000, 6, 100, 1), (30_000, 12, 300, 2), (7_000, 4, 200, 3), (20_000, 9, 150, 4)]


def _members():
    return [nw.structured_spec(n, p, k, seed) for n, p, k, seed in SPECS]


def _noise(specs, steps):
    return [lo.torch_noise_stream(10 + i, s.n, steps, False)[0] for i, s in enumerate(specs)]


@pytest.mark.parametrize("syn", [E.SYN_PUSH_EXACT, E.SYN_PULL])
def test_batch_equals_solo_runs(gpu, syn):
    specs = _members()
    steps = 500
    zs = _noise(specs, steps)
    solo = []
    for s, z in zip(specs, zs):
        with E.Engine.structured(s, pull=True) as eng:
            eng.set_noise_injected(z)
            r = eng.run(steps, vmean=True, record_spikes=True, syn_mode=syn)
            solo.append((r, eng.read_state(E.STATE_V), eng.read_state(E.STATE_J)))
    engines = [E.Engine.structured(s, pull=True) for s in specs]
    for e, z in zip(engines, zs):
        e.set_noise_injected(z)
    with E.Batch(engines) as b:
        got = b.run(200, vmean=True, record_spikes=True, syn_mode=syn)
        got2 = b.run(300, vmean=True, record_spikes=True, syn_mode=syn)
    for i, (r, v, j) in enumerate(solo):
        sp = np.concatenate([got[i].spikes, got2[i].spikes])
        assert np.array_equal(sp, r.spikes), f"member {i}"
        assert np.array_equal(np.concatenate([got[i].freqs, got2[i].freqs]), r.freqs)
        assert np.allclose(np.concatenate([got[i].vmeans, got2[i].vmeans]), r.vmeans, rtol=1e-6)
        assert np.array_equal(engines[i].read_state(E.STATE_V), v)
        assert np.array_equal(engines[i].read_state(E.STATE_J), j)
    assert any(r.spikes[300:].mean() > 0.005 for r, _, _ in solo)
    for e in engines:
        e.close()


def test_batch_graph_window_and_solo_interleave(gpu):
    """Float push: graph-replayed windows; members keep running on their own in between."""
    specs = _members()
    engines = [E.Engine.structured(s, seed=i) for i, s in enumerate(specs)]
    with E.Batch(engines) as b:
        b.run(800)                       # warm-up (tunes the push inside)
        for _ in range(3):               # a window shape is captured the third time in a row
            r1 = b.run(400)
        inf = b.info()
        assert inf["graph_launches"] >= 1
        solo = engines[1].run(100)       # a member alone between batch runs
        r2 = b.run(400)
    for i, e in enumerate(engines):
        assert e.info().step == 2400 + (100 if i == 1 else 0)
        rate1 = r1[i].freqs.sum() / (400 * specs[i].n)
        rate2 = r2[i].freqs.sum() / (400 * specs[i].n)
        assert rate1 > 0 and rate2 > 0
        assert abs(rate2 - rate1) < 0.5 * rate1
    assert solo.freqs.sum() > 0
    for e in engines:
        e.close()


@pytest.mark.parametrize("graph,param", [(False, 8), (True, 2008), (True, 2016)])
def test_batch_local_push_step(gpu, graph, param):
    """Batched population-local push: from saved mid-run member states, one float
    step gives every member the exact push's spikes and V, and J within float rounding."""
    specs = _members()
    engines = [E.Engine.structured(s, seed=i) for i, s in enumerate(specs)]
    assert all(e.info().local_windows > 0 for e in engines)
    with E.Batch(engines, graph=graph) as b:
        b.run(500, syn_mode=E.SYN_PUSH_EXACT)
        blobs = [e.save_state() for e in engines]
        ref = b.run(1, record_spikes=True, syn_mode=E.SYN_PUSH_EXACT)
        v_ref = [e.read_state(E.STATE_V) for e in engines]
        j_ref = [e.read_state(E.STATE_J) for e in engines]
        for e, blob in zip(engines, blobs):
            e.load_state(blob)
        b.set_push_variant(E.PUSH_LOCAL, param)
        got = b.run(1, record_spikes=True, syn_mode=E.SYN_PUSH)
        assert b.info()["push_kind"] == E.PUSH_LOCAL
    for i, e in enumerate(engines):
        assert np.array_equal(got[i].spikes, ref[i].spikes)
        assert np.array_equal(e.read_state(E.STATE_V), v_ref[i])
        assert np.allclose(e.read_state(E.STATE_J), j_ref[i], rtol=1e-5, atol=1e-5)
    assert sum(int(r.spikes.sum()) for r in ref) > 0
    for e in engines:
        e.close()


def test_batch_rejects_mixed_weight_types(gpu):
    a = E.Engine.structured(nw.structured_spec(3000, 3, 50, 1))
    b = E.Engine.structured(nw.structured_spec(3000, 3, 50, 2), weight_type=E.W_BF16)
    with pytest.raises(E.DtbError) as ei:
        E.Batch([a, b])
    assert ei.value.status == E.UNSUPPORTED
    a.close()
    b.close()
