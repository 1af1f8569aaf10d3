"""The snn.Snn gRPC front, end to end: a client speaking snn.proto drives the
engine through Init / Run / Update* / GetVersion / Shutdown, and every answer
equals a direct run of the same merged network through the C-ABI."""
import grpc
import numpy as np
import pytest

from dtb_b200 import engine as E
from dtb_b200 import network as nw
from dtb_b200 import server as S
from dtb_b200 import snn_pb2 as pb
from dtb_b200 import snn_pb2_grpc as pbg

pytestmark = pytest.mark.gpu


def _blocks(tmp_path):
    a = nw.make_uniform_block(3000, 40, seed=1)
    b = nw.make_uniform_block(2000, 40, seed=2)
    b["property"][:, 3] = np.repeat([0, 1], 1000)
    b["input_block_idx"] = b["input_block_idx"].copy()
    b["input_block_idx"][::7] = -1                      # some synapses come from block 0
    d = tmp_path / "single"
    d.mkdir()
    nw.write_npz(str(d / "block_0.npz"), a)
    nw.write_npz(str(d / "block_1.npz"), b)
    return str(d)


def _run(stub, **kw):
    return list(stub.Run(pb.RunRequest(**kw)))


def test_server_matches_direct_engine(gpu, tmp_path):
    path = _blocks(tmp_path)
    server, port, svc = S.start(0, syn_mode=E.SYN_PUSH_EXACT, seed=7)
    try:
        ch = grpc.insecure_channel(f"127.0.0.1:{port}")
        stub = pbg.SnnStub(ch)
        assert stub.GetVersion(pb.Empty()).version == 1000
        init = list(stub.Init(pb.InitRequest(file_path=path, delta_t=0.1)))
        assert [r.status for r in init] == [pb.SNN_OK, pb.SNN_OK]
        assert [r.neurons_per_block for r in init] == [3000, 2000]
        assert [(s.subblk_id, s.subblk_num) for s in init[1].subblk_info] == [(0, 1000), (1, 1000)]
        bad = _run(stub, iter=0)
        assert bad[0].status == pb.SNN_INVALID_PARAMETER
        bad = _run(stub, iter=5, output_sample_spike=True)
        assert bad[0].status == pb.SNN_UNSET_SAMPLE_FAILURE
        r1 = _run(stub, iter=300, output_freq=True, output_vmean=True, use_ou_background=True)
        # property surface, the way BlockWrapper sends it
        assert stub.Updateprop(iter([pb.UpdatePropRequest(block_id=1, neuron_id=[5, 6], prop_id=[pb.THRESHOLD_V] * 2,
                                                          prop_val=[-52.0, -52.0])])).success
        assert stub.Updatehyperpara(iter([pb.UpdateHyperParaRequest(block_id=1, prop_id=[pb.CONDUCT_G_AMPA],
                                                                    brain_id=[1], hpara_val=[1.2])])).success
        assert stub.Updateoubackgroundparam(iter([pb.UpdateOUBackgroundParamRequest(
            block_id=0, brain_id=[0], mean=[0.7], deviation=[0.25], correlation_time=[8.0])])).success
        assert stub.Updatesample(iter([pb.UpdateSampleRequest(block_id=0, sample_idx=[1, 2, 3]),
                                       pb.UpdateSampleRequest(block_id=1, sample_idx=[0, 7])])).success
        r2 = _run(stub, iter=200, output_freq=True, freq_char=True, use_ou_background=True,
                  output_sample_spike=True, output_sample_vmemb=True, output_imean=True,
                  output_receptor_imeas=True, output_sample_isynaptic=True)
        sub = _run(stub, iter=5, t_steps=2, use_ou_background=True, output_freq=True)   # substeps run
        assert len(sub) == 5 and all(r.status == pb.SNN_OK for r in sub)
        assert _run(stub, iter=5, t_steps=2, use_ou_background=False)[0].status == pb.SNN_INVALID_PARAMETER
        assert not stub.Updatedopaminecurrentparam(iter([pb.UpdateDopamineCurrentParamRequest(block_id=0)])).success
        assert stub.Shutdown(pb.ShutdownRequest()).shutdown
        ch.close()
    finally:
        server.stop(grace=1)
        svc.close()
    # the same sequence directly through the C-ABI
    net, blocks = S.merge_blocks(S._block_files(path))
    with E.Engine.from_arrays(net, seed=7) as eng:
        d1 = eng.run(300, vmean=True, syn_mode=E.SYN_PUSH_EXACT)
        eng.update_props([3005, 3006], [5, 5], [-52.0, -52.0])
        eng.update_prop_cols([7], [2], [1.2])
        eng.set_ou([0], [0.7], [0.25], [8.0])
        eng.set_samples([1, 2, 3, 3000, 3007])
        d2 = eng.run(200, syn_mode=E.SYN_PUSH_EXACT, sample_spike=True, sample_v=True, imean=True,
                     receptor_imean=True, sample_isyn=True)
        sizes = eng.pop_sizes.astype(np.float32)
    f1 = np.stack([np.frombuffer(r.freq[0], np.int32) for r in r1])
    v1 = np.stack([np.frombuffer(r.vmean[0], np.float32) for r in r1])
    assert np.array_equal(f1, d1.freqs) and np.array_equal(v1, d1.vmeans)
    assert f1.sum() > 0
    f2 = np.stack([np.frombuffer(r.freq[0], np.uint8) for r in r2])
    expect = np.floor(np.float32(255) * d2.freqs.astype(np.float32) / sizes + 0.5).astype(np.uint8)
    assert np.array_equal(f2, expect)
    s2 = np.stack([np.frombuffer(r.sample_spike[0], np.uint8) for r in r2])
    sv = np.stack([np.frombuffer(r.sample_vmemb[0], np.float32) for r in r2])
    assert np.array_equal(s2, d2.sample_spike) and np.array_equal(sv, d2.sample_v)
    im = np.stack([np.frombuffer(r.imean[0], np.float32) for r in r2])
    assert np.array_equal(im, d2.imeans)
    for c, name in enumerate(("ampa_imean", "nmda_imean", "gabaa_imean", "gabab_imean")):
        got = np.stack([np.frombuffer(getattr(r, name)[0], np.float32) for r in r2])
        assert np.array_equal(got, d2.receptor_imeans[:, c])
    si = np.stack([np.frombuffer(r.sample_isynaptic[0], np.float32) for r in r2])
    assert np.array_equal(si, d2.sample_isyn) and np.abs(si).max() > 0


def test_served_clients_share_the_gpu(gpu, tmp_path):
    """--serve: two client connections each Init their own network into the pool, and
    their Runs, issued from two threads, advance together on the GPU (continuous
    batching, fixed-point push).  Each client's counts equal its network run alone,
    including an Updateoubackgroundparam applied with the second client's Run."""
    import threading
    dirs = []
    for k in range(2):
        net = nw.make_uniform_block(20000 + 4000 * k, 100, seed=10 + k)
        net["property"][:, 3] = np.repeat([0, 1], [10000, 10000 + 4000 * k])
        d = tmp_path / f"client{k}" / "single"
        d.mkdir(parents=True)
        nw.write_npz(str(d / "block_0.npz"), net)
        dirs.append(str(d))
    server, port, svc = S.start(0, serve=True, slice_steps=50, seed=3)
    try:
        # two channels of one process share a connection (one peer) unless each keeps its own subchannels
        chans = [grpc.insecure_channel(f"127.0.0.1:{port}", options=[("grpc.use_local_subchannel_pool", 1)])
                 for _ in range(2)]
        stubs = [pbg.SnnStub(c) for c in chans]
        for st, d in zip(stubs, dirs):                   # sessions 0 and 1, in this order
            init = list(st.Init(pb.InitRequest(file_path=d, delta_t=0.1)))
            assert init[0].status == pb.SNN_OK and len(init[0].subblk_info) == 2
        assert len(svc.sessions) == 2                    # one session per connection
        assert stubs[1].Updateoubackgroundparam(iter([pb.UpdateOUBackgroundParamRequest(
            block_id=0, brain_id=[1], mean=[0.66], deviation=[0.22], correlation_time=[12.0])])).success
        assert not stubs[0].Updateprop(iter([pb.UpdatePropRequest(block_id=0, neuron_id=[1], prop_id=[5],
                                                                  prop_val=[-50.0])])).success
        bad = _run(stubs[0], iter=10, output_freq=True, output_vmean=True, use_ou_background=True)
        assert bad[0].status == pb.SNN_UNSUPPORTED
        got = [None, None]

        def client(k):
            r = _run(stubs[k], iter=4000, output_freq=True, use_ou_background=True)   # ~50 ms: the Runs overlap
            got[k] = np.array([np.frombuffer(x.freq[0], np.int32) for x in r])

        threads = [threading.Thread(target=client, args=(k,)) for k in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        info = svc.pool.info()
        assert info["n_nets"] == 2 and info["batch_members_sum"] > info["slices"]   # the Runs shared slices
        for k, d in enumerate(dirs):
            net, _ = S.merge_blocks(S._block_files(d))
            with E.Engine.from_arrays(net, seed=3 + k) as eng:
                if k == 1:
                    eng.set_ou(eng.pop_ids, np.float32([0.6, 0.66]), np.float32([0.2, 0.22]), np.float32([10.0, 12.0]))
                ref = eng.run(4000, syn_mode=E.SYN_PUSH_FIXED).freqs
            assert ref.sum() > 0
            assert np.array_equal(got[k], ref), f"client {k}"
        for c in chans:
            c.close()
    finally:
        server.stop(grace=1)
        svc.close()
