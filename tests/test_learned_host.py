"""Host-side logic of the learned parts (no GPU): the switch's prior fit,
the weight-file length check, and the policy argument checks that run
before any device call."""
import numpy as np
import pytest


def test_fit_prior_recovers_plane():
    from opengraph_b200.learned import PRIOR_INPUTS, SWITCH_BOUND, fit_prior, prior_of
    rng = np.random.default_rng(0)
    X = rng.normal(size=(5000, 8)).astype(np.float32)
    a = np.zeros(8)
    a[list(PRIOR_INPUTS)] = np.linspace(-1.0, 1.0, len(PRIOR_INPUTS)) + 0.1
    y = (X @ a + 2.5 + 0.01 * rng.normal(size=5000)).astype(np.float32)
    tail = fit_prior(X, y)
    assert tail.shape == (10,) and tail.dtype == np.float32
    assert np.allclose(tail[:8], a, atol=1e-2) and abs(tail[8] - 2.5) < 1e-2
    assert all(tail[i] == 0 for i in range(8) if i not in PRIOR_INPUTS) and tail[9] == SWITCH_BOUND
    assert np.abs(prior_of(tail, X) - y).max() < 0.1


def test_switch_blob_length(lib, tmp_path, monkeypatch):
    import opengraph_b200 as og
    from opengraph_b200 import learned
    n = og.mlp_nparams(lib, 8, 64)
    assert n == 4801
    monkeypatch.setattr(learned, "WEIGHTS", str(tmp_path))
    np.zeros(n, np.float32).tofile(tmp_path / learned.SWITCH[0])      # the network without its prior
    with pytest.raises(ValueError):
        learned.load_weights(lib, learned.SWITCH)
    np.zeros(n + 10, np.float32).tofile(tmp_path / learned.SWITCH[0])
    assert len(learned.load_weights(lib, learned.SWITCH)) == n + 10
    assert learned.load_weights(lib, ("absent.f32", 8, 64, 10)) is None


def test_set_policy_rejects_bad_prior(lib):
    import opengraph_b200 as og
    p = np.zeros(og.mlp_nparams(lib, 8, 64) + 10, np.float32)
    for i, v in ((-1, -1.0), (-2, np.nan), (-5, np.inf)):   # negative bound, non-finite bias / coefficient
        q = p.copy()
        q[i] = v
        assert lib.ogb_bfs_set_policy(q.ctypes.data) != 0
