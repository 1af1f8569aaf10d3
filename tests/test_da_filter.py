"""Data-assimilation filter (DA_voxel.filter, data_assimilation/DA_voxel.py:289-307):
the CPU restatement against the reference's own update, and the CUDA kernels
(dtb_da_filter) against both."""
import importlib.util
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.bold_oracle import da_filter

_spec = importlib.util.spec_from_file_location("make_da_golden", os.path.join(GOLDEN, "make_da_golden.py"))
_gen = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_gen)


def _golden():
    g = np.load(os.path.join(GOLDEN, "da_filter.npz"))
    w_hat, y, noise = _gen.inputs(int(g["e"]), int(g["v"]), int(g["hp"]), int(g["seed"]))
    return g, w_hat, y, noise


def test_oracle_against_reference_golden():
    g, w_hat, y, noise = _golden()
    w = da_filter(w_hat, y, noise, int(g["hp"]), float(g["sigma"]), float(g["rate"]))
    assert np.abs(g["w"] - w_hat).max() > 1e-2            # the update moves the state
    assert np.allclose(w, g["w"], rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
def test_filter_kernel_against_oracle_and_golden(gpu):
    import torch
    from dtb_b200 import engine as E
    g, w_hat, y, noise = _golden()
    out = E.da_filter(torch.from_numpy(w_hat).cuda(), torch.from_numpy(y).cuda(), torch.from_numpy(noise).cuda(),
                      float(g["sigma"]), float(g["rate"])).cpu().numpy()
    ref = da_filter(w_hat, y, noise, int(g["hp"]), float(g["sigma"]), float(g["rate"]))
    assert np.allclose(out, ref, rtol=1e-6, atol=1e-7)
    assert np.allclose(out, g["w"], rtol=1e-6, atol=1e-6)
    # a DA-sized problem: 100 members x 1000 voxels, 10 states
    w2, y2, n2 = _gen.inputs(100, 1000, 4, 9)
    out2 = E.da_filter(torch.from_numpy(w2).cuda(), torch.from_numpy(y2).cuda(), torch.from_numpy(n2).cuda(), 1e-6, 0.5)
    assert np.allclose(out2.cpu().numpy(), da_filter(w2, y2, n2, 4, 1e-6, 0.5), rtol=1e-6, atol=1e-7)
