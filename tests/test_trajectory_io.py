"""Trajectory files in the reference's Saver format: written here, read by the reference's loader."""
import os
import sys

import numpy as np
import pytest
import torch

from fvm_solver_b200 import trajectory_io as tio

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))


def test_snapshot_round_trip_and_keys(tmp_path):
    g = torch.Generator().manual_seed(0)
    prims = torch.randn(500, 4, generator=g) * torch.tensor([3.0, 0.5, 0.05, 4.0]) + torch.tensor([3.0, 0, 1, 100])
    bc = prims[:40] + 0.01
    path = tio.write_snapshot(str(tmp_path), 0.125, prims, bc)
    assert os.path.basename(path) == "t_0.125.npz"
    d = np.load(path)
    assert sorted(d.files) == ["bc_primatives", "cell_primatives", "prim_mean", "prim_std", "t"]
    assert d["cell_primatives"].dtype == np.float16 and d["prim_mean"].shape == (1, 4)
    t, cell, bcl = tio.load_step(path)
    assert float(t) == 0.125
    assert torch.allclose(cell, prims, rtol=0, atol=float(prims.std(0).max()) * 2e-3)
    assert torch.allclose(bcl, bc, rtol=0, atol=float(prims.std(0).max()) * 2e-3)


def test_reference_loader_reads_our_files(tmp_path):
    from refimport import import_reference, reference_available
    if not reference_available():
        pytest.skip("reference sources not present")
    import importlib
    import_reference()
    saving = importlib.import_module("time_fvm.ds_saving.saving")
    prims = torch.randn(300, 4)
    path = tio.write_snapshot(str(tmp_path), 2.5, prims, prims[:10])
    t_ref, cell_ref, bc_ref = saving.load_step(path)
    t, cell, bc = tio.load_step(path)
    assert float(t_ref) == float(t) and torch.equal(cell_ref, cell) and torch.equal(bc_ref, bc)
