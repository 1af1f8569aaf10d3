"""BOLD signal (data assimilation, models/bold_model_pytorch.py:61-96): the CPU
restatement against the reference model's own output, and the CUDA kernel
(dtb_bold_run) against both."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.bold_oracle import DA_PARAMS, BoldOracle, bold_inputs

# float32 powf results differ by an ulp between math libraries; everything else
# follows the same float32 operation order
REL = 2e-6


def _golden():
    return np.load(os.path.join(GOLDEN, "bold_da_params.npz"))


def test_oracle_against_reference_golden():
    g = _golden()
    n, steps, every = int(g["n"]), int(g["steps"]), int(g["every"])
    u = bold_inputs(n, steps, int(g["seed"]))
    o = BoldOracle(*DA_PARAMS.values(), n=n)
    outs = []
    for s in range(steps):
        x = o.run(u[s])
        if s % every == every - 1:
            outs.append(x)
    outs = np.array(outs)
    assert np.max(np.abs(outs - g["out"]) / np.abs(g["out"])) < REL
    assert np.allclose(o.state(), g["state"], rtol=REL, atol=1e-7)
    assert g["out"].min() > 0.0 and np.ptp(g["out"]) > 1e-3


@pytest.mark.gpu
def test_bold_kernel_against_oracle_and_golden(gpu):
    import torch
    from dtb_b200 import engine as E
    g = _golden()
    n, steps, every = int(g["n"]), int(g["steps"]), int(g["every"])
    u = torch.from_numpy(bold_inputs(n, steps, int(g["seed"]))).cuda()
    state = torch.tensor(np.stack([np.zeros(n), np.zeros(n), np.ones(n), np.ones(n)]), dtype=torch.float32).cuda()
    # two windows of 800 steps, the way DA advances one assimilation window at a time
    out = torch.cat([E.bold_run(u[:800], state), E.bold_run(u[800:], state)]).cpu().numpy()
    torch.cuda.synchronize()
    sel = out[every - 1::every]
    assert np.max(np.abs(sel - g["out"]) / np.abs(g["out"])) < REL
    assert np.allclose(state.cpu().numpy(), g["state"], rtol=REL, atol=1e-7)
    o = BoldOracle(*DA_PARAMS.values(), n=n)
    ref = np.array([o.run(x) for x in u.cpu().numpy()])
    assert np.max(np.abs(out - ref) / np.abs(ref)) < REL
    # a larger ensemble x voxel grid, state only (out=None), against the oracle
    n2 = 100 * 230
    u2 = torch.from_numpy(bold_inputs(n2, 200, 3)).cuda()
    st2 = torch.tensor(np.stack([np.zeros(n2), np.zeros(n2), np.ones(n2), np.ones(n2)]), dtype=torch.float32).cuda()
    assert E.bold_run(u2, st2, out=False) is None
    o2 = BoldOracle(*DA_PARAMS.values(), n=n2)
    for x in u2.cpu().numpy():
        o2.run(x)
    assert np.allclose(st2.cpu().numpy(), o2.state(), rtol=REL, atol=1e-7)
