"""Ensembles on the device: models advanced concurrently on their own streams give the same
results as each model advanced alone (no shared scratch, no cross-stream races)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_concurrent_ensemble_matches_models_alone():
    from meeuuw_b200.ensemble import Ensemble, sample_configs
    from meeuuw_b200.timestep import GPUModel
    cfgs = sample_configs(5, seed=11, n_range=(16, 32), Ra_range=(1e4, 1e5), contrast_range=(1.0, 1e3))
    ens = Ensemble(cfgs, stokes="mixed", threads=4)
    for _ in range(3):
        ens.step()
    ens.synchronize()
    ens.check()
    got = ens.diagnostics()
    states = [(m.T.cpu().numpy(), m.x.cpu().numpy()) for m in ens.models]
    ens.close()
    for cfg, d, (T, x) in zip(cfgs, got, states):
        m = GPUModel(cfg, stokes="mixed")
        for _ in range(3):
            m.step()
        ref = m.diagnostics()
        assert d["stokes"]["converged"] == 1
        assert np.array_equal(T, m.T.cpu().numpy()) and np.array_equal(x, m.x.cpu().numpy()), cfg.name
        assert d["vrms"] == ref["vrms"] and d["Nu"] == ref["Nu"], (cfg.name, d, ref)
