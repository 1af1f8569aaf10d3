"""The reference's own client drives the gRPC front unchanged.

``python/dist_blockwrapper.py`` (``BlockWrapper``) is loaded from the reference
checkout named by ``DTB_REFERENCE`` (skipped when unset; nothing of it is copied
here) and talks to ``server.py`` over a real gRPC channel, exactly as
``data_assimilation/DA_voxel.py:309-353, 418`` drives ``dist_simulator``: Init of a
two-block directory (with the client's population-id rebasing,
dist_blockwrapper.py:77-120), ``run`` with freqs / freq_char / vmean / imean /
receptor imeans / samples and the OU background, ``update_property``,
``mul_property_by_subblk``, ``assign_property_by_subblk``,
``gamma_property_by_subblk``, ``update_ou_background_stimuli``, ``set_samples``
and ``get_version``.  The server runs on the CPU stand-in engine built on the
oracle (tests/oracle_engine.py), and every tensor the client decodes is checked
against a second stand-in driven directly with the same calls.

Two adaptations for a host without a GPU or with the client's own slips: the
client keeps its tensors on CUDA (``.cuda()`` at class definition and in every
method), which here leaves them on the CPU; and ``gamma_property_by_subblk`` reads
a module global ``debug`` that the client never defines, set here to False.
"""
import importlib.util
import os
import sys
import types

import numpy as np
import pytest
import torch

from dtb_b200 import network as nw
from dtb_b200 import server as srv
from dtb_b200 import snn_pb2, snn_pb2_grpc
from tests.oracle_engine import OracleEngine

REF_ROOT = os.environ.get("DTB_REFERENCE", "")
CLIENT = os.path.join(REF_ROOT, "python", "dist_blockwrapper.py") if REF_ROOT else ""
pytestmark = pytest.mark.skipif(not CLIENT or not os.path.exists(CLIENT),
                                reason="DTB_REFERENCE names no reference checkout with python/dist_blockwrapper.py")

SEED = 5
# the client's property-column -> PropType table (dist_blockwrapper.py:32)
COL_TO_PROP = [19, -1, 0, -1, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18]


@pytest.fixture
def client_module(monkeypatch):
    monkeypatch.setattr(torch.Tensor, "cuda", lambda self, *a, **k: self)
    pkg = types.ModuleType("dtb_reference_client")
    pkg.__path__ = []
    names = ["dtb_reference_client", "dtb_reference_client.snn_pb2", "dtb_reference_client.snn_pb2_grpc",
             "dtb_reference_client.dist_blockwrapper"]
    monkeypatch.setitem(sys.modules, names[0], pkg)
    monkeypatch.setitem(sys.modules, names[1], snn_pb2)
    monkeypatch.setitem(sys.modules, names[2], snn_pb2_grpc)
    spec = importlib.util.spec_from_file_location(names[3], CLIENT)
    mod = importlib.util.module_from_spec(spec)
    monkeypatch.setitem(sys.modules, names[3], mod)
    spec.loader.exec_module(mod)
    mod.debug = False
    return mod


def _blocks(tmp_path):
    """Two blocks of two populations each (ids 0 and 1 in both), with synapses across."""
    rng = np.random.default_rng(2)
    sizes = [1200, 900]
    files = []
    d = tmp_path / "net" / "single"
    os.makedirs(d)
    for b, n in enumerate(sizes):
        prop = nw.lif_property(n, np.repeat([0, 1], [n // 2, n - n // 2]))
        k_local, k_far = 60, 20
        post = np.repeat(np.arange(n, dtype=np.uint32), k_local + k_far)
        pre = np.concatenate([np.concatenate([rng.integers(0, n, k_local), rng.integers(0, sizes[1 - b], k_far)])
                              for _ in range(n)]).astype(np.uint32)
        blk = np.tile(np.concatenate([np.zeros(k_local), np.full(k_far, 1 - 2 * b)]), n).astype(np.int16)
        kind = (rng.random(pre.size) < 0.2).astype(np.uint8) * 2
        w = rng.random((pre.size, 2), dtype=np.float32)
        f = str(d / f"block_{b}.npz")
        np.savez(f, property=prop, input_block_idx=blk, input_neuron_idx=pre, output_neuron_idx=post,
                 input_channel_offset=kind, weight=w)
        files.append(f)
    return str(d), files


def test_blockwrapper_drives_the_server(tmp_path, client_module):
    path, files = _blocks(tmp_path)
    server, port, svc = srv.start(0, engine_factory=OracleEngine, seed=SEED)
    try:
        bw = client_module.BlockWrapper(f"127.0.0.1:{port}", path, 0.1)
        net, blocks = srv.merge_blocks(files)
        ref = OracleEngine(net, dt=0.1, seed=SEED)
        # Init: four populations, the second block's ids rebased by the client to 2 and 3
        assert bw.subblk_id.tolist() == [0, 1, 2, 3]
        assert bw.neurons_per_subblk.tolist() == [600, 600, 450, 450]
        assert bw.total_neurons.item() == 2100
        assert bw.get_version() == "Version: 1.0.0"

        def run(n, **kw):
            out = list(bw.run(n, **kw))
            return [torch.stack([o[k] for o in out]).numpy() for k in range(len(out[0]))] if isinstance(out[0], tuple) \
                else torch.stack(out).numpy()

        # the OU background per population (update_ou_background_stimuli), then a run with every mean output
        bw.update_ou_background_stimuli(torch.tensor([1, 3]), torch.tensor([10.0, 12.0]), torch.tensor([0.62, 0.58]),
                                        torch.tensor([0.2, 0.25]))
        ref.set_ou([1, 3], np.float32([0.62, 0.58]), np.float32([0.2, 0.25]), np.float32([10.0, 12.0]))
        fr, vm, im, a, nmda, ga, gb = run(300, freqs=True, vmean=True, imean=True, receptor_imean=True, iou=True)
        r = ref.run(300, freq=True, vmean=True, imean=True, receptor_imean=True)
        assert r.freqs[100:].sum() > 0
        assert np.array_equal(fr, r.freqs)
        assert np.array_equal(vm, r.vmeans) and np.array_equal(im, r.imeans)
        for c, got in enumerate((a, nmda, ga, gb)):
            assert np.array_equal(got, r.receptor_imeans[:, c])

        # per-neuron properties (update_property: [global neuron, property column])
        idx = torch.tensor([[5, 8], [1500, 8], [7, 2]], dtype=torch.int64)
        val = torch.tensor([-52.0, -51.0, 0.3], dtype=torch.float32)
        bw.update_property(idx, val)
        ref.update_props([5, 1500, 7], [COL_TO_PROP[8], COL_TO_PROP[8], COL_TO_PROP[2]], [-52.0, -51.0, 0.3])
        # per-population multiply and assign (mul / assign_property_by_subblk: [subblock id, column])
        bw.mul_property_by_subblk(torch.tensor([[0, 10], [3, 12]]), torch.tensor([1.2, 0.9]))
        ref.update_prop_cols([COL_TO_PROP[10], COL_TO_PROP[12]], [0, 3], [1.2, 0.9])
        bw.assign_property_by_subblk(torch.tensor([[2, 11]]), torch.tensor([0.0025]))
        ref.update_prop_cols([COL_TO_PROP[11]], [2], [0.0025], assign=True)
        # Gamma draws per population (gamma_property_by_subblk)
        bw.gamma_property_by_subblk(torch.tensor([[1, 10]]), torch.tensor([4.0]), torch.tensor([400.0]))
        ref.update_gamma([COL_TO_PROP[10]], [1], [4.0], [400.0])
        assert np.array_equal(svc.eng.prop, ref.prop)

        # freq_char: the client turns the bytes back into counts (count / n * 255 -> count)
        ch = run(200, freqs=True, freq_char=True, iou=True)
        r = ref.run(200, freq=True)
        assert np.abs(ch - r.freqs).max() <= np.ceil(bw.neurons_per_subblk.numpy().max() / 255.0)

        # samples in the client's own order, across both blocks
        sample = torch.tensor([1800, 3, 1200, 40, 999], dtype=torch.int64)
        bw.set_samples(sample)
        ref.set_samples(np.sort(sample.numpy()))
        sp, v, iou = run(100, freqs=False, output_sample_spike=True, output_sample_vmemb=True,
                         output_sample_iou=True, iou=True)
        r = ref.run(100, freq=False, sample_spike=True, sample_v=True, sample_iou=True)
        order = np.argsort(np.argsort(sample.numpy()))      # the client's recover order
        assert np.array_equal(sp, r.sample_spike[:, order])
        assert np.array_equal(v, r.sample_v[:, order]) and np.array_equal(iou, r.sample_iou[:, order])
        bw.close()
    finally:
        server.stop(grace=1)
        svc.close()
