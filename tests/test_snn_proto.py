"""The snn.proto contract (runtime-built descriptors) and the block merge of the server."""
import os
import re

import numpy as np
import pytest

from dtb_b200 import network as nw
from dtb_b200 import snn_pb2 as pb

# the reference checkout, when one is named (e.g. DTB_REFERENCE=/path/to/Digital_twin_brain-open)
REF_ROOT = os.environ.get("DTB_REFERENCE", "")
REF_PROTO = os.path.join(REF_ROOT, "protos", "snn.proto") if REF_ROOT else ""
_TYPES = {"int32": pb.T_INT32, "float": pb.T_FLOAT, "double": pb.T_DOUBLE, "bool": pb.T_BOOL,
          "string": pb.T_STRING, "bytes": pb.T_BYTES}


def test_messages_round_trip():
    r = pb.RunRequest(iter=800, t_steps=1, output_freq=True, freq_char=True, use_ou_background=True)
    assert pb.RunRequest.FromString(r.SerializeToString()) == r
    q = pb.UpdatePropRequest(block_id=1, neuron_id=[3, 4], prop_id=[pb.THRESHOLD_V, 19], prop_val=[-52.0, 0.1])
    assert list(pb.UpdatePropRequest.FromString(q.SerializeToString()).prop_id) == [5, 19]
    i = pb.InitRequest(file_path="/x/single", delta_t=0.1, mode=pb.InitRequest.CommMode.COMM_ROUTE)
    assert pb.InitRequest.FromString(i.SerializeToString()).mode == 1
    assert pb.SnnStatus.SNN_OK == 0 and pb.SnnStatus.SNN_INVALID_NETWORK == 5
    assert pb.PropType.NOISE_RATE == 19


@pytest.mark.skipif(not REF_PROTO or not os.path.exists(REF_PROTO), reason="DTB_REFERENCE names no reference checkout")
def test_descriptor_matches_reference_proto():
    """Every message field (name, number, type, label) equals protos/snn.proto's."""
    text = re.sub(r"//.*", "", open(REF_PROTO).read())
    enums = set(re.findall(r"enum\s+(\w+)", text))
    for mname, body in re.findall(r"message\s+(\w+)\s*\{((?:[^{}]|\{[^{}]*\})*)\}", text):
        body = re.sub(r"enum\s+\w+\s*\{[^{}]*\}", "", body)
        fields = re.findall(r"(repeated\s+)?(\w+)\s+(\w+)\s*=\s*(\d+)\s*;", body)
        ours = {f[0]: f for f in pb.MESSAGES[mname]}
        assert len(fields) == len(ours), mname
        for rep, ftype, fname, num in fields:
            name, number, t, label, tname = ours[fname]
            assert number == int(num), (mname, fname)
            assert label == (pb.REP if rep else pb.ONE), (mname, fname)
            if ftype in _TYPES:
                assert t == _TYPES[ftype], (mname, fname)
            elif ftype in enums or ftype == "CommMode":
                assert t == pb.T_ENUM and tname.endswith(ftype), (mname, fname)
            else:
                assert t == pb.T_MSG and tname.endswith(ftype), (mname, fname)
    rpcs = re.findall(r"rpc\s+(\w+)\s*\(\s*(stream\s+)?(\w+)\s*\)\s*returns\s*\(\s*(stream\s+)?(\w+)\s*\)", text)
    assert [(n, q, bool(cs), r, bool(ss)) for n, cs, q, ss, r in rpcs] == [(m[0], m[1], m[3], m[2], m[4])
                                                                          for m in pb.METHODS]


def test_grpc_stub_has_every_rpc():
    import grpc
    from dtb_b200 import snn_pb2_grpc as pbg
    ch = grpc.insecure_channel("127.0.0.1:1")
    stub = pbg.SnnStub(ch)
    for name, *_ in pb.METHODS:
        assert callable(getattr(stub, name))
    ch.close()


def test_merge_blocks_makes_one_network(tmp_path):
    """Two blocks with cross-block synapses become one network with absolute ids."""
    import importlib
    server = importlib.import_module("dtb_b200.server")
    a = nw.make_uniform_block(300, 10, seed=1)
    b = nw.make_uniform_block(200, 10, seed=2)
    b["property"][:, 3] = np.repeat([0, 1], 100)
    # block 1's first 50 synapses come from block 0 (relative block id -1)
    b["input_block_idx"] = b["input_block_idx"].copy()
    b["input_block_idx"][:50] = -1
    d = tmp_path / "single"
    d.mkdir()
    nw.write_npz(str(d / "block_0.npz"), a)
    nw.write_npz(str(d / "block_1.npz"), b)
    net, blocks = server.merge_blocks(server._block_files(str(d)))
    assert net["property"].shape == (500, 22)
    assert [blk["offset"] for blk in blocks] == [0, 300]
    assert blocks[1]["subblk"] == [(0, 100), (1, 100)]
    assert list(np.unique(net["property"][:, 3])) == [0, 1, 2]
    pre = net["input_neuron_idx"].astype(np.int64)
    post = net["output_neuron_idx"].astype(np.int64)
    sa = a["input_neuron_idx"].size
    assert np.array_equal(pre[:sa], a["input_neuron_idx"])
    assert np.array_equal(pre[sa:sa + 50], b["input_neuron_idx"][:50])            # from block 0
    assert np.array_equal(pre[sa + 50:], 300 + b["input_neuron_idx"][50:].astype(np.int64))
    assert np.array_equal(post[sa:], 300 + b["output_neuron_idx"].astype(np.int64))
    assert server._weight_type(str(d / "block_0.npz"), np.float32) == 0
