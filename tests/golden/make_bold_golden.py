"""Generate the BOLD golden vectors by running the reference's own model.

Runs ``models/bold_model_pytorch.py`` (``BOLD.run``, torch float32 on the CPU) from
the reference checkout (NOT shipped with this repository) with DA_voxel.py's
parameters on ``oracle.bold_oracle.bold_inputs(128, 1600, seed=1)`` and records
the signal of every 4th step and the final state (s, q, v, f_in).

Usage (needs the reference checkout; a few seconds):
    python tests/golden/make_bold_golden.py /path/to/Digital_twin_brain-open
"""
import importlib.util
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.bold_oracle import DA_PARAMS, bold_inputs  # noqa: E402

N, STEPS, SEED, EVERY = 128, 1600, 1, 4


def main(ref_root):
    spec = importlib.util.spec_from_file_location("bold_model_ref", os.path.join(ref_root, "models", "bold_model_pytorch.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    torch.set_num_threads(1)
    b = mod.BOLD(DA_PARAMS["epsilon"], DA_PARAMS["tao_s"], DA_PARAMS["tao_f"], DA_PARAMS["tao_0"], DA_PARAMS["alpha"],
                 DA_PARAMS["E_0"], DA_PARAMS["V_0"])
    u = bold_inputs(N, STEPS, SEED)
    outs = []
    for s in range(STEPS):
        o = b.run(torch.from_numpy(u[s]))
        if s % EVERY == EVERY - 1:
            outs.append(o.numpy().copy())
    state = torch.stack([b.s, b.q, b.v, b.f_in]).numpy()
    path = os.path.join(HERE, "bold_da_params.npz")
    np.savez_compressed(path, out=np.array(outs), state=state, n=np.array(N), steps=np.array(STEPS),
                        seed=np.array(SEED), every=np.array(EVERY))
    print("->", path, os.path.getsize(path) // 1024, "KB")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DTB_REFERENCE", ""))
