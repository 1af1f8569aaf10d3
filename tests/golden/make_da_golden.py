"""Generate the DA-filter golden vectors by running the reference's own update.

Extracts ``DA_Task_V1.filter`` from ``data_assimilation/DA_voxel.py`` of the
reference checkout (NOT shipped with this repository; the method is taken from
the source with ``ast`` because the module's other imports -- its gRPC client,
plotting and table libraries -- are not needed for it), runs it with torch
float32 on the CPU on seeded inputs (``torch.normal`` replaced by fixed draws, so
the model noise is reproducible) and records the updated state.

Usage (needs the reference checkout; a second):
    python tests/golden/make_da_golden.py /path/to/Digital_twin_brain-open
"""
import ast
import os
import sys
import textwrap
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
E, V, HP, SIGMA, RATE, SEED = 64, 48, 4, 1e-6, 0.5, 3


def inputs(e=E, v=V, hp=HP, seed=SEED):
    """Seeded filter inputs: the ensemble state w_hat [E, V, hp + 6], the observation, the noise draws."""
    rng = np.random.default_rng(seed)
    w_hat = (1.0 + 0.1 * rng.standard_normal((e, v, hp + 6))).astype(np.float32)
    y = (1.0 + 0.05 * rng.standard_normal(v)).astype(np.float32)
    noise = rng.standard_normal((e, v)).astype(np.float32)
    return w_hat, y, noise


def main(ref_root):
    src = open(os.path.join(ref_root, "data_assimilation", "DA_voxel.py")).read()
    fn = None
    for node in ast.walk(ast.parse(src)):
        if isinstance(node, ast.ClassDef) and node.name == "DA_Task_V1":
            for b in node.body:
                if isinstance(b, ast.FunctionDef) and b.name == "filter":
                    fn = ast.get_source_segment(src, b)
    ns = {"torch": torch}
    exec(textwrap.dedent(fn), ns)
    w_hat, y, noise = inputs()
    self = types.SimpleNamespace(hp_num=HP, ensembles=E, bold_sigma=SIGMA)
    normal = torch.normal
    torch.normal = lambda mean, std, size: torch.from_numpy(noise)
    try:
        w = ns["filter"](self, torch.from_numpy(w_hat), torch.from_numpy(y), rate=RATE).numpy()
    finally:
        torch.normal = normal
    path = os.path.join(HERE, "da_filter.npz")
    np.savez_compressed(path, w=w, e=np.array(E), v=np.array(V), hp=np.array(HP), sigma=np.array(SIGMA),
                        rate=np.array(RATE), seed=np.array(SEED))
    print("->", path, os.path.getsize(path) // 1024, "KB")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DTB_REFERENCE", ""))
