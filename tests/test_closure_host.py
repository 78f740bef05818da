"""Host side of the learned closure: the parameter layout shared by the C
API, the numpy oracle and the training driver, and the weights file."""

from __future__ import annotations

import numpy as np

from oracle import closure_oracle as CO
from polesitter_b200 import closure as CL


def test_parameter_layout_matches_the_oracle_and_the_header():
    assert CL.N_PARAMS == CO.N_PARAMS == 9928
    header = open(CL.os.path.join(CL.HERE, "..", "include", "polesitter_b200.h")).read()
    assert "#define PS_B200_CLOSURE_PARAMS 9928" in header


def test_init_params_padding_is_zero():
    p = CL.init_params(7)
    parts = CO.unpack(p)
    assert np.all(parts["W1"][13:] == 0)
    assert np.all(parts["W4"][:, 3:] == 0)
    assert np.all(parts["b1"] == 0) and np.all(parts["b4"] == 0)
    assert np.abs(parts["W2"]).max() > 0
    assert np.array_equal(p, CL.init_params(7))


def test_shipped_weights_load(tmp_path):
    params, meta = CL.load(CL.default_weights_path())
    assert params.shape == (CL.N_PARAMS,) and np.all(np.isfinite(params))
    assert meta["theta"] > 0 and meta["n"] >= 1024
    assert meta["eval_median_mlp"] < meta["eval_median_base"]
    parts = CO.unpack(params)
    assert np.all(parts["W1"][13:] == 0) and np.all(parts["W4"][:, 3:] == 0)
    path = tmp_path / "w.npz"
    CL.save(str(path), params, theta=7.0, n=1024)
    p2, m2 = CL.load(str(path))
    assert np.array_equal(p2, params) and m2["theta"] == 7.0


def test_oracle_features_are_scale_free():
    # scaling every mass (hence L and G) by k leaves the network inputs
    # unchanged and scales the correction's scale factor by k
    rng = np.random.default_rng(0)
    raw = rng.normal(size=(50, 16)).astype(np.float32)
    raw[:, 12] = np.abs(raw[:, 12]) + 0.1
    raw[:, 13] = rng.integers(1, 11, 50)
    raw[:, 14] = np.abs(raw[:, 14]) + 0.01
    x, s = CO.features_from_raw(raw)
    scaled = raw.copy()
    scaled[:, 0:9] *= 8.0
    x2, s2 = CO.features_from_raw(scaled)
    assert np.allclose(x, x2, atol=1e-6)
    assert np.allclose(s2, 8.0 * s, rtol=1e-6)
