"""GPU test of the learned closure's training pipeline on a small case:
fine run -> explicit filters of two widths -> dimensionless features and
targets -> Adam on the tensor cores -> a-priori check on held-out
snapshots.  It shows what the trained network gains over the method
without it: at each filter width, the held-out correlation and normalised
MSE of the deviatoric SGS stresses with the filtered truth, network vs the
Deardorff eddy viscosity evaluated with the filtered SGS energy."""
import argparse
import importlib.util
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _tc():
    spec = importlib.util.spec_from_file_location(
        "train_closure", os.path.join(ROOT, "paes-channelflow_b200", "train_closure.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_trained_network_beats_deardorff_a_priori(gpu_lib, tmp_path):
    tc = _tc()
    a = argparse.Namespace(fine=[128, 128, 64], factors=[2, 4], re_tau=395.0, snapshots=24, spinup=2000, every=20,
                           amp=1.0, large=0.3, spinup_precision=4, seed=7, holdout=0.25, epochs=6, batch=16384,
                           lr=1e-3, out=str(tmp_path / "sgs"))
    rep = tc.run(a, log=lambda *x: None)
    comps = list(tc.COMPONENTS)
    for fac in ("2", "4"):
        ap = rep["apriori_heldout"][fac]
        rho_net = np.array([ap[c]["network"]["rho"] for c in comps])
        rho_dd = np.array([ap[c]["deardorff"]["rho"] for c in comps])
        mse_net = np.array([ap[c]["network"]["nmse"] for c in comps])
        mse_dd = np.array([ap[c]["deardorff"]["nmse"] for c in comps])
        assert rho_net.mean() > rho_dd.mean() + 0.1, (fac, rho_net, rho_dd)
        assert (mse_net < mse_dd).sum() >= 5, (fac, mse_net, mse_dd)
        assert ap["dissipation"]["network"] > 0  # the runtime sign test would use the network
    loss = rep["training"]["loss"]
    assert loss[-1][1] < loss[0][1]
    z = np.load(str(tmp_path / "sgs.npz"))
    assert z["params"].shape == (9478,) and z["norm"].shape == (34,)
