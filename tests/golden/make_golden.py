"""Generate the golden vectors by running the reference's own CPU model.

Runs ``models/block_new.py`` from the reference checkout (NOT shipped with this
repository) on the plain 10,000-neuron block and records, per case:

* ``spikes``: the threshold spikes of every step, ``np.packbits`` of [steps, N];
* ``mean_act`` [steps] and ``mean_psc`` [steps, 4]: block_new's per-population
  outputs (one population);
* ``v_trace`` [steps, 64]: V of 64 fixed neurons at every step;
* ``v_full_<s>`` [N]: V of every neuron after step s, for a few s;
* ``j_full_<s>`` [4, N]: the receptor accumulators after step s;
* ``digest``: sha256 of the generated network, so a regenerated network is
  checked to be the one the golden run used.

Usage (needs the reference checkout; runs ~1 minute on 8 cores):
    python tests/golden/make_golden.py /path/to/Digital_twin_brain-open
"""
import importlib.util
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

N, K, STEPS = 10_000, 100, 1000
SAMPLE = np.linspace(0, N - 1, 64).astype(np.int64)
FULL_AT = (1, 2, 5, 10, 50, 100, 300, 1000)
CASES = {
    # name: (dyadic weights, debug_mode, noise_rate)
    "threshold": (False, False, 0.0),
    "noise": (False, True, 0.01),
    "threshold_dyadic": (True, False, 0.0),
    "noise_dyadic": (True, True, 0.01),
}


def load_module(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def dense_w(net, n):
    w = torch.zeros(4, n, n)
    ch = torch.from_numpy(np.where(net["input_channel_offset"] != 0, 2, 0).astype(np.int64))
    post = torch.from_numpy(net["output_neuron_idx"].astype(np.int64))
    pre = torch.from_numpy(net["input_neuron_idx"].astype(np.int64))
    wt = torch.from_numpy(net["weight"])
    w.index_put_((ch, post, pre), wt[:, 0], accumulate=True)
    w.index_put_((ch + 1, post, pre), wt[:, 1], accumulate=True)
    return w


def main(ref_root):
    block_new = load_module(os.path.join(ref_root, "models", "block_new.py"), "block_new_ref")
    network = load_module(os.path.join(ROOT, "digital_twin_brain-open_b200", "network.py"), "dtb_network")
    torch.set_num_threads(os.cpu_count())
    for name, (dyadic, debug, rate) in CASES.items():
        net = network.make_uniform_block(N, K, seed=0, noise_rate=rate, dyadic_weights=dyadic)
        w = dense_w(net, N)
        torch.manual_seed(0)
        b = block_new.block(torch.from_numpy(net["property"]), w, delta_t=0.1,
                            i_mean=0.6, i_sigma=0.2, tau_i=10.0)
        spikes = np.zeros((STEPS, N), bool)
        mean_act = np.zeros(STEPS, np.float32)
        mean_psc = np.zeros((STEPS, 4), np.float32)
        v_trace = np.zeros((STEPS, len(SAMPLE)), np.float32)
        out = {}
        for s in range(STEPS):
            act, psc = b.run(debug, rate)
            spikes[s] = b.active.numpy()
            mean_act[s] = act.numpy()[0]
            mean_psc[s] = psc.numpy()[0]
            v_trace[s] = b.V_i.numpy()[SAMPLE]
            if s + 1 in FULL_AT:
                out[f"v_full_{s + 1}"] = b.V_i.numpy().copy()
                out[f"j_full_{s + 1}"] = b.J_ui.numpy().copy()
        out.update(spikes=np.packbits(spikes, axis=1), mean_act=mean_act, mean_psc=mean_psc,
                   v_trace=v_trace, sample=SAMPLE, digest=np.array(network.arrays_digest(net)),
                   steps=np.array(STEPS), n=np.array(N), k=np.array(K), noise_rate=np.array(rate),
                   debug=np.array(debug), dyadic=np.array(dyadic), seed=np.array(0))
        path = os.path.join(HERE, f"block_new_{name}.npz")
        np.savez_compressed(path, **out)
        print(name, "rate Hz", spikes.mean() * 1e4, "->", path, os.path.getsize(path) // 1024, "KB")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DTB_REFERENCE", ""))
