"""gRPC ``snn.Snn`` server over the B200 engine (the reference's
tools/dist_simulator.cpp master + workers, for one GPU).

``python digital_twin_brain-open_b200/server.py --port 50051`` serves the
``snn.proto`` contract so python/dist_blockwrapper.py (and data_assimilation/
DA_voxel.py through it) drive the engine unchanged.

Init loads every ``block_<i>.npz`` of the directory (the reference gives one to
each MPI rank, dist_simulator.cpp:1368) and merges them into ONE network resident
in this GPU: block b's neurons follow blocks 0..b-1; a synapse's presynaptic
neuron is ``offset[b + input_block_idx] + input_neuron_idx`` (the relative block
id is made absolute as adjust_relative_conn_bid does, src/configuration.cpp:956);
each (block, population id) pair becomes one population.  Every RPC keeps the
reference's per-block addressing: neuron ids relative to their block, population
(``brain_id``) ids as the block's own subblock ids, responses in block order.

``--serve``: many clients share the GPU.  Each client connection (gRPC peer) Inits
its own network, resident in a pool under an HBM cap (``dtb_server_*``); Run
requests of all clients go to the pool's online scheduler, which batches the
requests in flight slice by slice (continuous batching) with the deterministic
fixed-point push, so each client's counts are the same as its network run alone.
Served Runs carry the OU background and output_freq / freq_char;
Updateoubackgroundparam is applied with the client's next Run; the other outputs
and property updates answer SNN_UNSUPPORTED / success = False in this mode.
A session is keyed by the connection's peer address: gRPC Python channels of one
process to the same target share one connection unless they are created with the
channel option ``grpc.use_local_subchannel_pool``, so two clients in one process
need that option (or separate processes) to hold separate networks.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import glob
import math
import os
import re
import shutil
import tempfile
import threading

import grpc
import numpy as np

from . import engine as E
from . import snn_pb2 as pb
from . import snn_pb2_grpc as pbg

VERSION = 1 * 1000 + 0 * 100 + 0   # include/version.hpp: major*1000 + minor*100 + patch


def _block_files(path):
    if os.path.isfile(path):
        return [path]
    files = glob.glob(os.path.join(path, "block_*.npz"))
    key = lambda f: int(re.search(r"block_(\d+)\.npz$", f).group(1))  # noqa: E731
    return sorted(files, key=key)


def _weight_type(path, dtype):
    """The reference picks the weight type from the directory name (configuration.cpp:1411-1435)."""
    for sub, wt in (("/double", E.W_F64), ("/single", E.W_F32), ("/half", E.W_F16), ("/int8", E.W_U8),
                    ("/uint8", E.W_U8)):
        if sub in path:
            return wt
    return {np.dtype(np.float64): E.W_F64, np.dtype(np.float32): E.W_F32, np.dtype(np.float16): E.W_F16,
            np.dtype(np.uint8): E.W_U8}[np.dtype(dtype)]


def merge_blocks(files):
    """Load the block files and merge them into one network in the npz key set.

    Returns (network dict, blocks) with blocks[b] = dict(offset, n, subblk=[(id, count)], pop_ids=[global ids]).
    """
    raw = [dict(np.load(f)) for f in files]
    sizes = [r["property"].shape[0] for r in raw]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    props, pre, post, kind, w, blocks = [], [], [], [], [], []
    next_pop = 0
    for b, r in enumerate(raw):
        p = r["property"].astype(np.float32).copy()
        col = p[:, 3]
        starts = np.concatenate([[0], np.nonzero(col[1:] != col[:-1])[0] + 1])
        ends = np.concatenate([starts[1:], [len(col)]])
        subblk, gids = [], []
        for s, e in zip(starts, ends):
            subblk.append((int(col[s]), int(e - s)))
            gids.append(next_pop)
            p[s:e, 3] = next_pop
            next_pop += 1
        props.append(p)
        blocks.append(dict(offset=int(offsets[b]), n=sizes[b], subblk=subblk, pop_ids=gids,
                           by_subblk={sid: [g for (sid2, _), g in zip(subblk, gids) if sid2 == sid]
                                      for sid, _ in subblk}))
        if r["input_neuron_idx"].size:
            rel = r.get("input_block_idx", np.zeros(r["input_neuron_idx"].shape[0], np.int16)).astype(np.int64)
            src_block = b + rel
            if (src_block < 0).any() or (src_block >= len(raw)).any():
                raise ValueError(f"block {b}: input_block_idx points outside the {len(raw)} blocks")
            pre.append(offsets[src_block] + r["input_neuron_idx"].astype(np.int64))
            post.append(offsets[b] + r["output_neuron_idx"].astype(np.int64))
            kind.append(r["input_channel_offset"].astype(np.uint8))
            w.append(r["weight"])
    cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dt)  # noqa: E731
    net = dict(property=np.concatenate(props), input_neuron_idx=cat(pre, np.uint32),
               output_neuron_idx=cat(post, np.uint32), input_channel_offset=cat(kind, np.uint8),
               weight=np.concatenate(w) if w else np.zeros((0, 2), np.float32))
    return net, blocks


class SnnService(pbg.SnnServicer):
    """The ``snn.Snn`` service backed by one engine."""

    def __init__(self, syn_mode=E.SYN_PUSH, device_weight=None, seed=0, chunk=1000, stop_event=None,
                 engine_factory=None, serve=False, hbm_cap_gb=150.0, slice_steps=100):
        """``engine_factory(net, **options)`` builds the engine of an Init (default
        ``engine.Engine.from_arrays``, the CUDA engine); a test can hand in another
        object with the same methods.  ``serve``: one network per client in a pool
        with continuous batching (module docstring)."""
        self.engine_factory = engine_factory or E.Engine.from_arrays
        self.serve = serve
        self.sessions = {}
        if serve:
            self.pool = E.Server(hbm_cap_bytes=hbm_cap_gb * 1e9, slice_steps=slice_steps, syn_mode=E.SYN_PUSH_FIXED)
            self.pool.start(E.SERVE_BATCHED)
            self.pool_dir = tempfile.mkdtemp(prefix="dtb_pool_")
        self.syn_mode = syn_mode
        self.device_weight = device_weight
        self.seed = seed
        self.chunk = chunk
        self.eng = None
        self.blocks = []
        self.iterations = 0
        self.lock = threading.Lock()
        self.stop_event = stop_event or threading.Event()
        self.n_samples = 0

    # ---- helpers
    def _global_pops(self, block_id, brain_ids, blocks=None):
        b = (self.blocks if blocks is None else blocks)[block_id]
        out, idx = [], []
        for k, sid in enumerate(brain_ids):
            for g in b["by_subblk"].get(int(sid), []):
                out.append(g)
                idx.append(k)
        return np.asarray(out, np.uint32), np.asarray(idx, np.int64)

    # ---- RPCs
    def GetVersion(self, request, context):
        return pb.Version(version=VERSION)

    def Init(self, request, context):
        if self.serve:
            yield from self._init_served(request, context)
            return
        with self.lock:
            if not request.file_path:
                yield pb.InitResponse(status=pb.SNN_INVALID_PARAMETER)
                return
            files = _block_files(request.file_path)
            if not files:
                yield pb.InitResponse(status=pb.SNN_INVALID_NETWORK)
                return
            net, blocks = merge_blocks(files)
            if not any(b["subblk"] for b in blocks):
                yield pb.InitResponse(status=pb.SNN_INVALID_NETWORK)
                return
            in_wt = _weight_type(request.file_path, net["weight"].dtype)
            dev_wt = self.device_weight
            if dev_wt is None:
                dev_wt = {E.W_F64: E.W_F32, E.W_F32: E.W_F32, E.W_F16: E.W_F16, E.W_U8: E.W_U8}[in_wt]
            if self.eng is not None:
                self.eng.close()
            self.eng = self.engine_factory(net, dt=request.delta_t or 1.0, weight_type=dev_wt, seed=self.seed,
                                           push=self.syn_mode != E.SYN_PULL, pull=self.syn_mode == E.SYN_PULL)
            self.blocks = blocks
            self.iterations = 0
            self.n_samples = 0
            for b, blk in enumerate(blocks):
                yield pb.InitResponse(status=pb.SNN_OK, block_id=b, neurons_per_block=blk["n"],
                                      subblk_info=[pb.SubblockInfo(subblk_id=s, subblk_num=c) for s, c in blk["subblk"]],
                                      total_gpu_mem=float(self.eng.info().device_bytes))

    # ---- serving mode: one network per client connection in the pool
    def _init_served(self, request, context):
        with self.lock:
            if not request.file_path:
                yield pb.InitResponse(status=pb.SNN_INVALID_PARAMETER)
                return
            files = _block_files(request.file_path)
            if not files:
                yield pb.InitResponse(status=pb.SNN_INVALID_NETWORK)
                return
            net, blocks = merge_blocks(files)
            if not any(b["subblk"] for b in blocks):
                yield pb.InitResponse(status=pb.SNN_INVALID_NETWORK)
                return
            in_wt = _weight_type(request.file_path, net["weight"].dtype)
            dev_wt = self.device_weight if self.device_weight is not None else \
                {E.W_F64: E.W_F32, E.W_F32: E.W_F32, E.W_F16: E.W_F16, E.W_U8: E.W_U8}[in_wt]
            # the pool rebuilds evicted networks from a file: the merged network, written once
            k = len(self.sessions)
            path = os.path.join(self.pool_dir, f"net_{k}.npz")
            nw_arrays = dict(net, input_block_idx=np.zeros(net["input_neuron_idx"].shape[0], np.int16))
            np.savez(path, **nw_arrays)
            P = sum(len(b["subblk"]) for b in blocks)
            self.pool.stop()                          # networks join the pool between scheduler runs
            try:
                nid = self.pool.add_npz(path, P, dt=request.delta_t or 1.0, weight_type=dev_wt, seed=self.seed + k)
            finally:
                self.pool.start(E.SERVE_BATCHED)
            self.sessions[context.peer()] = dict(net=nid, blocks=blocks, P=P, counts=np.concatenate(
                [[c for _, c in b["subblk"]] for b in blocks]).astype(np.float32),
                ou=[np.full(P, 0.6, np.float32), np.full(P, 0.2, np.float32), np.full(P, 10.0, np.float32)],
                ou_dirty=False)
            for b, blk in enumerate(blocks):
                yield pb.InitResponse(status=pb.SNN_OK, block_id=b, neurons_per_block=blk["n"],
                                      subblk_info=[pb.SubblockInfo(subblk_id=s, subblk_num=c) for s, c in blk["subblk"]],
                                      total_gpu_mem=0.0)

    def _run_served(self, request, context):
        sess = self.sessions.get(context.peer())
        status = pb.SNN_OK
        if sess is None:
            status = pb.SNN_INVALID_NETWORK
        elif request.iter <= 0 or (request.t_steps > 1 and not request.use_ou_background):
            status = pb.SNN_INVALID_PARAMETER
        elif (request.output_vmean or request.output_sample_spike or request.output_sample_vmemb or
              request.output_sample_iou or request.output_sample_isynaptic or request.output_imean or
              request.output_receptor_imeas or request.t_steps > 1 or not request.use_ou_background):
            status = pb.SNN_UNSUPPORTED
        if status != pb.SNN_OK:
            yield pb.RunResponse(status=status)
            return
        ou = None
        if sess["ou_dirty"]:
            ou, sess["ou_dirty"] = tuple(a.copy() for a in sess["ou"]), False
        ticket = self.pool.submit(sess["net"], request.iter, ou)
        r = self.pool.wait(ticket)
        if r["status"] != E.OK:
            yield pb.RunResponse(status=pb.SNN_INVALID_PARAMETER)
            return
        for k in range(request.iter):
            resp = pb.RunResponse(status=pb.SNN_OK)
            if request.output_freq:
                f = r["freqs"][k]
                if request.freq_char:
                    q = (np.float32(255) * f.astype(np.float32)) / sess["counts"]
                    resp.freq.append(np.array([math.floor(x + 0.5) for x in q], np.uint8).tobytes())
                else:
                    resp.freq.append(f.astype(np.int32).tobytes())
            yield resp

    def Run(self, request, context):
        if self.serve:
            yield from self._run_served(request, context)
            return
        # validation of SnnImpl::Run (dist_simulator.cpp:3225-3234)
        samples_wanted = (request.output_sample_spike or request.output_sample_vmemb or request.output_sample_iou
                          or request.output_sample_isynaptic)
        status = pb.SNN_OK
        if self.eng is None:
            status = pb.SNN_INVALID_NETWORK
        elif request.iter <= 0:
            status = pb.SNN_INVALID_PARAMETER
        elif samples_wanted and self.n_samples == 0:
            status = pb.SNN_UNSET_SAMPLE_FAILURE
        elif request.output_sample_iou and not request.use_ou_background:
            status = pb.SNN_INVALID_PARAMETER
        elif request.t_steps > 1 and not request.use_ou_background:
            status = pb.SNN_INVALID_PARAMETER
        elif request.t_steps > 255 or (request.t_steps > 1 and self.syn_mode == E.SYN_PULL):
            status = pb.SNN_UNSUPPORTED     # substeps need a push mode; at most 255 per step
        elif ((request.output_imean or request.output_receptor_imeas or request.output_sample_isynaptic)
              and self.syn_mode == E.SYN_PULL):
            status = pb.SNN_UNSUPPORTED     # the pull kernel completes J one step later
        if status != pb.SNN_OK:
            yield pb.RunResponse(status=status)
            return
        with self.lock:
            counts = self.eng.pop_sizes.astype(np.float32)
            done = 0
            while done < request.iter:
                it = min(self.chunk, request.iter - done)
                r = self.eng.run(it, use_ou=request.use_ou_background, freq=request.output_freq,
                                 vmean=request.output_vmean, syn_mode=self.syn_mode,
                                 sample_spike=request.output_sample_spike, sample_v=request.output_sample_vmemb,
                                 sample_iou=request.output_sample_iou, imean=request.output_imean,
                                 receptor_imean=request.output_receptor_imeas,
                                 sample_isyn=request.output_sample_isynaptic, t_steps=max(1, request.t_steps))
                for k in range(it):
                    resp = pb.RunResponse(status=pb.SNN_OK)
                    if request.output_freq:
                        f = r.freqs[k]
                        if request.freq_char:
                            # lroundf(float(255 * count) / float(n)), stat_result.cpp:128
                            q = (np.float32(255) * f.astype(np.float32)) / counts
                            resp.freq.append(np.array([math.floor(x + 0.5) for x in q], np.uint8).tobytes())
                        else:
                            resp.freq.append(f.astype(np.int32).tobytes())
                    if request.output_vmean:
                        resp.vmean.append(r.vmeans[k].astype(np.float32).tobytes())
                    if request.output_sample_spike:
                        resp.sample_spike.append(r.sample_spike[k].tobytes())
                    if request.output_sample_vmemb:
                        resp.sample_vmemb.append(r.sample_v[k].tobytes())
                    if request.output_sample_iou:
                        resp.sample_iou.append(r.sample_iou[k].tobytes())
                    if request.output_sample_isynaptic:
                        resp.sample_isynaptic.append(r.sample_isyn[k].tobytes())
                    if request.output_imean:
                        resp.imean.append(r.imeans[k].astype(np.float32).tobytes())
                    if request.output_receptor_imeas:
                        ri = r.receptor_imeans[k]
                        resp.ampa_imean.append(ri[0].tobytes())
                        resp.nmda_imean.append(ri[1].tobytes())
                        resp.gabaa_imean.append(ri[2].tobytes())
                        resp.gabab_imean.append(ri[3].tobytes())
                    yield resp
                done += it
            self.iterations += request.iter

    def Updateprop(self, request_iterator, context):
        if self.serve:                      # not part of the served path
            for _ in request_iterator:
                pass
            return pb.UpdatePropResponse(success=False)
        with self.lock:
            for req in request_iterator:
                b = self.blocks[req.block_id]
                nid = np.asarray(req.neuron_id, np.int64) + b["offset"]
                self.eng.update_props(nid, np.asarray(req.prop_id, np.uint32), np.asarray(req.prop_val, np.float32))
        return pb.UpdatePropResponse(success=True)

    def Updatehyperpara(self, request_iterator, context):
        if self.serve:                      # not part of the served path
            for _ in request_iterator:
                pass
            return pb.UpdateHyperParaResponse(success=False)
        with self.lock:
            for req in request_iterator:
                pops, k = self._global_pops(req.block_id, req.brain_id)
                if pops.size:
                    self.eng.update_prop_cols(np.asarray(req.prop_id, np.uint32)[k], pops,
                                              np.asarray(req.hpara_val, np.float32)[k], assign=req.assigned)
        return pb.UpdateHyperParaResponse(success=True)

    def Updategamma(self, request_iterator, context):
        if self.serve:                      # not part of the served path
            for _ in request_iterator:
                pass
            return pb.UpdateGammaResponse(success=False)
        with self.lock:
            for req in request_iterator:
                pops, k = self._global_pops(req.block_id, req.brain_id)
                if pops.size:
                    self.eng.update_gamma(np.asarray(req.prop_id, np.uint32)[k], pops,
                                          np.asarray(req.gamma_concentration, np.float32)[k],
                                          np.asarray(req.gamma_rate, np.float32)[k])
        return pb.UpdateGammaResponse(success=True)

    def Updateoubackgroundparam(self, request_iterator, context):
        if self.serve:
            # kept with the client's session and applied with its next Run
            sess = self.sessions.get(context.peer())
            for req in request_iterator:
                if sess is None:
                    continue
                pops, k = self._global_pops(req.block_id, req.brain_id, sess["blocks"])
                for arr, vals in zip(sess["ou"], (req.mean, req.deviation, req.correlation_time)):
                    arr[pops] = np.asarray(vals, np.float32)[k]
                sess["ou_dirty"] = True
            return pb.UpdateOUBackgroundParamResponse(success=sess is not None)
        with self.lock:
            for req in request_iterator:
                pops, k = self._global_pops(req.block_id, req.brain_id)
                if pops.size:
                    self.eng.set_ou(pops, np.asarray(req.mean, np.float32)[k], np.asarray(req.deviation, np.float32)[k],
                                    np.asarray(req.correlation_time, np.float32)[k])
        return pb.UpdateOUBackgroundParamResponse(success=True)

    def Updatesample(self, request_iterator, context):
        if self.serve:                      # not part of the served path
            for _ in request_iterator:
                pass
            return pb.UpdateSampleResponse(success=False)
        with self.lock:
            ids = []
            for req in request_iterator:
                ids.append(np.asarray(req.sample_idx, np.int64) + self.blocks[req.block_id]["offset"])
            ids = np.concatenate(ids) if ids else np.zeros(0, np.int64)
            self.eng.set_samples(ids)
            self.n_samples = int(ids.size)
        return pb.UpdateSampleResponse(success=True)

    # currents outside the LIF path (T-type Ca, dopamine, adaptation) are not part of this engine
    def Updatettypecacurrentparam(self, request_iterator, context):
        for _ in request_iterator:
            pass
        return pb.UpdateTTypeCaCurrentParamResponse(success=False)

    def Updatedopaminecurrentparam(self, request_iterator, context):
        for _ in request_iterator:
            pass
        return pb.UpdateDopamineCurrentParamResponse(success=False)

    def Updateadaptationcurrentparam(self, request_iterator, context):
        for _ in request_iterator:
            pass
        return pb.UpdateAdaptationCurrentParamResponse(success=False)

    def Shutdown(self, request, context):
        self.stop_event.set()
        return pb.ShutdownResponse(shutdown=True)

    def close(self):
        if self.eng is not None:
            self.eng.close()
            self.eng = None
        if self.serve and self.pool is not None:
            self.pool.close()
            self.pool = None
            shutil.rmtree(self.pool_dir, ignore_errors=True)


def start(port=0, host="127.0.0.1", **kw):
    """Start a server; returns (server, bound port, service)."""
    stop = threading.Event()
    svc = SnnService(stop_event=stop, **kw)
    max_len = 2 ** 31 - 1
    server = grpc.server(concurrent.futures.ThreadPoolExecutor(max_workers=4),
                         options=[("grpc.max_send_message_length", max_len),
                                  ("grpc.max_receive_message_length", max_len)])
    pbg.add_SnnServicer_to_server(svc, server)
    bound = server.add_insecure_port(f"{host}:{port}")
    server.start()
    return server, bound, svc


def main():
    ap = argparse.ArgumentParser(description="snn.Snn gRPC server on one B200")
    ap.add_argument("--port", type=int, default=50051)
    ap.add_argument("--host", default="0.0.0.0")
    ap.add_argument("--syn", default="push", choices=["push", "push_exact", "pull"])
    ap.add_argument("--bf16", action="store_true", help="store weights as bf16 pairs on the device")
    ap.add_argument("--serve", action="store_true",
                    help="one network per client connection, Runs batched on the GPU (continuous batching)")
    ap.add_argument("--hbm-cap-gb", type=float, default=150.0, help="HBM cap of the resident networks (--serve)")
    ap.add_argument("--slice-steps", type=int, default=100, help="steps per continuous-batching slice (--serve)")
    args = ap.parse_args()
    syn = {"push": E.SYN_PUSH, "push_exact": E.SYN_PUSH_EXACT, "pull": E.SYN_PULL}[args.syn]
    server, port, svc = start(args.port, args.host, syn_mode=syn, device_weight=E.W_BF16 if args.bf16 else None,
                              serve=args.serve, hbm_cap_gb=args.hbm_cap_gb, slice_steps=args.slice_steps)
    print(f"snn.Snn serving on {args.host}:{port}", flush=True)
    svc.stop_event.wait()
    server.stop(grace=2)
    svc.close()


if __name__ == "__main__":
    main()
