"""Message classes of the ``snn`` gRPC contract (protos/snn.proto), built at run time.

The reference generates ``snn_pb2.py`` from ``protos/snn.proto`` with
grpc_tools (gencode.sh:2-3); protoc is not available here, so the same
contract -- package ``snn``, every message, enum, field name, number, type and
label of protos/snn.proto:1-219 -- is declared below as a table and turned into
a ``FileDescriptorProto``.  The module exposes the same names the generated one
does (message classes, ``SnnStatus``, ``PropType`` and their values), so
``from .snn_pb2 import *`` in python/dist_blockwrapper.py:11 resolves unchanged.
"""
from google.protobuf import descriptor_pb2, descriptor_pool, message_factory
from google.protobuf.internal import enum_type_wrapper

_F = descriptor_pb2.FieldDescriptorProto
T_INT32, T_FLOAT, T_DOUBLE, T_BOOL, T_STRING, T_BYTES, T_ENUM, T_MSG = (
    _F.TYPE_INT32, _F.TYPE_FLOAT, _F.TYPE_DOUBLE, _F.TYPE_BOOL, _F.TYPE_STRING, _F.TYPE_BYTES, _F.TYPE_ENUM,
    _F.TYPE_MESSAGE)
ONE, REP = _F.LABEL_OPTIONAL, _F.LABEL_REPEATED

ENUMS = {
    "SnnStatus": ["SNN_OK", "SNN_INVALID_PARAMETER", "SNN_UNSET_SAMPLE_FAILURE", "SNN_UNSUPPORTED",
                  "SNN_NOT_ENABLE_METRIC", "SNN_INVALID_NETWORK"],
    "PropType": ["EXT_STIMULI_I", "MEMBRANE_C", "REF_T", "LEAKAGE_G", "LEAKAGE_V", "THRESHOLD_V", "RESET_V",
                 "CONDUCT_G_AMPA", "CONDUCT_G_NMDA", "CONDUCT_G_GABAa", "CONDUCT_G_GABAb", "MEMBRANE_V_AMPA",
                 "MEMBRANE_V_NMDA", "MEMBRANE_V_GABAa", "MEMBRANE_V_GABAb", "TAO_AMPA", "TAO_NMDA", "TAO_GABAa",
                 "TAO_GABAb", "NOISE_RATE"],
}

# message -> [(field, number, type, label, type name)], in protos/snn.proto order
MESSAGES = {
    "Empty": [],
    "Version": [("version", 1, T_INT32, ONE, None)],
    "InitRequest": [("file_path", 1, T_STRING, ONE, None), ("delta_t", 2, T_FLOAT, ONE, None),
                    ("mode", 3, T_ENUM, ONE, ".snn.InitRequest.CommMode")],
    "SubblockInfo": [("subblk_id", 1, T_INT32, ONE, None), ("subblk_num", 2, T_INT32, ONE, None)],
    "InitResponse": [("status", 1, T_ENUM, ONE, ".snn.SnnStatus"), ("block_id", 2, T_INT32, ONE, None),
                     ("neurons_per_block", 3, T_INT32, ONE, None),
                     ("subblk_info", 4, T_MSG, REP, ".snn.SubblockInfo"),
                     ("used_cpu_mem", 5, T_DOUBLE, ONE, None), ("total_gpu_mem", 6, T_DOUBLE, ONE, None),
                     ("used_gpu_mem", 7, T_DOUBLE, ONE, None)],
    "RunRequest": [("iter", 1, T_INT32, ONE, None), ("iter_offset", 2, T_INT32, ONE, None),
                   ("t_steps", 3, T_INT32, ONE, None), ("output_freq", 4, T_BOOL, ONE, None),
                   ("freq_char", 5, T_BOOL, ONE, None), ("output_vmean", 6, T_BOOL, ONE, None),
                   ("output_imean", 7, T_BOOL, ONE, None), ("use_ou_background", 8, T_BOOL, ONE, None),
                   ("output_receptor_imeas", 9, T_BOOL, ONE, None), ("output_sample_spike", 10, T_BOOL, ONE, None),
                   ("output_sample_vmemb", 11, T_BOOL, ONE, None), ("output_sample_iou", 12, T_BOOL, ONE, None),
                   ("output_sample_isynaptic", 13, T_BOOL, ONE, None)],
    "RunResponse": [("status", 1, T_ENUM, ONE, ".snn.SnnStatus"), ("freq", 2, T_BYTES, REP, None),
                    ("vmean", 3, T_BYTES, REP, None), ("sample_spike", 4, T_BYTES, REP, None),
                    ("sample_vmemb", 5, T_BYTES, REP, None), ("sample_iou", 6, T_BYTES, REP, None),
                    ("sample_isynaptic", 7, T_BYTES, REP, None), ("imean", 8, T_BYTES, REP, None),
                    ("ampa_imean", 9, T_BYTES, REP, None), ("nmda_imean", 10, T_BYTES, REP, None),
                    ("gabaa_imean", 11, T_BYTES, REP, None), ("gabab_imean", 12, T_BYTES, REP, None)],
    "UpdatePropRequest": [("block_id", 1, T_INT32, ONE, None), ("neuron_id", 2, T_INT32, REP, None),
                          ("prop_id", 3, T_ENUM, REP, ".snn.PropType"), ("prop_val", 4, T_FLOAT, REP, None)],
    "UpdatePropResponse": [("success", 1, T_BOOL, ONE, None)],
    "UpdateGammaRequest": [("block_id", 1, T_INT32, ONE, None), ("prop_id", 2, T_ENUM, REP, ".snn.PropType"),
                           ("brain_id", 3, T_INT32, REP, None), ("gamma_concentration", 4, T_FLOAT, REP, None),
                           ("gamma_rate", 5, T_FLOAT, REP, None)],
    "UpdateGammaResponse": [("success", 1, T_BOOL, ONE, None)],
    "UpdateHyperParaRequest": [("block_id", 1, T_INT32, ONE, None), ("prop_id", 2, T_ENUM, REP, ".snn.PropType"),
                               ("brain_id", 3, T_INT32, REP, None), ("hpara_val", 4, T_FLOAT, REP, None),
                               ("assigned", 5, T_BOOL, ONE, None)],
    "UpdateHyperParaResponse": [("success", 1, T_BOOL, ONE, None)],
    "UpdateSampleRequest": [("block_id", 1, T_INT32, ONE, None), ("sample_idx", 2, T_INT32, REP, None)],
    "UpdateSampleResponse": [("success", 1, T_BOOL, ONE, None)],
    "UpdateOUBackgroundParamRequest": [("block_id", 1, T_INT32, ONE, None), ("brain_id", 2, T_INT32, REP, None),
                                       ("mean", 3, T_FLOAT, REP, None), ("deviation", 4, T_FLOAT, REP, None),
                                       ("correlation_time", 5, T_FLOAT, REP, None)],
    "UpdateOUBackgroundParamResponse": [("success", 1, T_BOOL, ONE, None)],
    "UpdateTTypeCaCurrentParamRequest": [("block_id", 1, T_INT32, ONE, None), ("brain_id", 2, T_INT32, REP, None),
                                         ("h_init", 3, T_FLOAT, REP, None), ("g_t", 4, T_FLOAT, REP, None),
                                         ("tao_h_minus", 5, T_FLOAT, REP, None), ("tao_h_plus", 6, T_FLOAT, REP, None),
                                         ("v_h", 7, T_FLOAT, REP, None), ("v_t", 8, T_FLOAT, REP, None)],
    "UpdateTTypeCaCurrentParamResponse": [("success", 1, T_BOOL, ONE, None)],
    "UpdateDopamineCurrentParamRequest": [("block_id", 1, T_INT32, ONE, None), ("brain_id", 2, T_INT32, REP, None),
                                          ("v_da", 3, T_FLOAT, REP, None), ("g_da", 4, T_FLOAT, REP, None)],
    "UpdateDopamineCurrentParamResponse": [("success", 1, T_BOOL, ONE, None)],
    "UpdateAdaptationCurrentParamRequest": [("block_id", 1, T_INT32, ONE, None), ("brain_id", 2, T_INT32, REP, None),
                                            ("ca_init", 3, T_FLOAT, REP, None), ("ca_decay", 4, T_FLOAT, REP, None),
                                            ("alpha_constant", 5, T_FLOAT, REP, None), ("v_k", 6, T_FLOAT, REP, None),
                                            ("g_ahp", 7, T_FLOAT, REP, None)],
    "UpdateAdaptationCurrentParamResponse": [("success", 1, T_BOOL, ONE, None)],
    "ShutdownRequest": [],
    "ShutdownResponse": [("shutdown", 1, T_BOOL, ONE, None)],
}

# rpc name -> (request, response, client streaming, server streaming), protos/snn.proto:5-18
METHODS = [
    ("GetVersion", "Empty", "Version", False, False),
    ("Init", "InitRequest", "InitResponse", False, True),
    ("Run", "RunRequest", "RunResponse", False, True),
    ("Updateprop", "UpdatePropRequest", "UpdatePropResponse", True, False),
    ("Updategamma", "UpdateGammaRequest", "UpdateGammaResponse", True, False),
    ("Updatehyperpara", "UpdateHyperParaRequest", "UpdateHyperParaResponse", True, False),
    ("Updatesample", "UpdateSampleRequest", "UpdateSampleResponse", True, False),
    ("Updateoubackgroundparam", "UpdateOUBackgroundParamRequest", "UpdateOUBackgroundParamResponse", True, False),
    ("Updatettypecacurrentparam", "UpdateTTypeCaCurrentParamRequest", "UpdateTTypeCaCurrentParamResponse", True,
     False),
    ("Updatedopaminecurrentparam", "UpdateDopamineCurrentParamRequest", "UpdateDopamineCurrentParamResponse", True,
     False),
    ("Updateadaptationcurrentparam", "UpdateAdaptationCurrentParamRequest", "UpdateAdaptationCurrentParamResponse",
     True, False),
    ("Shutdown", "ShutdownRequest", "ShutdownResponse", False, False),
]


def _file_descriptor_proto():
    f = descriptor_pb2.FileDescriptorProto(name="snn.proto", package="snn", syntax="proto3")
    for name, values in ENUMS.items():
        e = f.enum_type.add(name=name)
        for i, v in enumerate(values):
            e.value.add(name=v, number=i)
    for name, fields in MESSAGES.items():
        m = f.message_type.add(name=name)
        if name == "InitRequest":
            e = m.enum_type.add(name="CommMode")
            e.value.add(name="COMM_P2P", number=0)
            e.value.add(name="COMM_ROUTE", number=1)
        for fname, num, ftype, label, tname in fields:
            fd = m.field.add(name=fname, number=num, type=ftype, label=label)
            if tname:
                fd.type_name = tname
    s = f.service.add(name="Snn")
    for name, req, resp, cs, ss in METHODS:
        s.method.add(name=name, input_type=f".snn.{req}", output_type=f".snn.{resp}", client_streaming=cs,
                     server_streaming=ss)
    return f


_POOL = descriptor_pool.DescriptorPool()
_POOL.Add(_file_descriptor_proto())
DESCRIPTOR = _POOL.FindFileByName("snn.proto")

for _name in MESSAGES:
    globals()[_name] = message_factory.GetMessageClass(DESCRIPTOR.message_types_by_name[_name])
for _name, _values in ENUMS.items():
    globals()[_name] = enum_type_wrapper.EnumTypeWrapper(DESCRIPTOR.enum_types_by_name[_name])
    for _i, _v in enumerate(_values):
        globals()[_v] = _i
COMM_P2P, COMM_ROUTE = 0, 1

__all__ = list(MESSAGES) + list(ENUMS) + [v for vs in ENUMS.values() for v in vs] + ["DESCRIPTOR"]
