"""A whole time step recorded as one CUDA graph (Stokes and energy loops as conditional nodes)
replays to exactly the states of eager steps, and ensembles of recorded steps match models
stepped alone."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _state(m):
    return [t.cpu().numpy().copy() for t in (m.T, m.x, m.z, m.solV, m.solP, m.u, m.w)]


@pytest.mark.parametrize("stokes", ["mixed", "f64"])
def test_recorded_step_replays_eager_steps(stokes):
    from meeuuw_b200 import configs
    from meeuuw_b200.timestep import GPUModel
    cfg = configs.fk_convection(32, seed=5, Ra=1e5)
    host = configs.build_host_model(cfg)
    a = GPUModel(cfg, host, stokes=stokes)
    b = GPUModel(cfg, host, stokes=stokes)
    for _ in range(4):
        a.step()
    b.step()
    b.capture_step()
    for _ in range(3):
        b.step()
    da, db = a.diagnostics(), b.diagnostics()
    for xa, xb in zip(_state(a), _state(b)):
        assert np.array_equal(xa, xb)
    assert da["vrms"] == db["vrms"] and da["Nu"] == db["Nu"] and da["dt"] == db["dt"]
    for k in ("outer_iters", "inner_iters", "refinements", "converged"):
        assert da["stokes"][k] == db["stokes"][k], (k, da["stokes"], db["stokes"])
    assert b.energy_info[0] == a.energy_info[0]


def test_recorded_ensemble_matches_models_alone():
    from meeuuw_b200.ensemble import Ensemble, sample_configs
    from meeuuw_b200.timestep import GPUModel
    cfgs = sample_configs(4, seed=13, n_range=(16, 32), Ra_range=(1e4, 1e5), contrast_range=(1.0, 1e3))
    ens = Ensemble(cfgs, stokes="mixed", graphs=True)
    for _ in range(3):
        ens.step()
    ens.synchronize()
    assert all(ens.active)
    got = [_state(m) for m in ens.models]
    diag = ens.diagnostics()
    ens.close()
    for cfg, st, d in zip(cfgs, got, diag):
        m = GPUModel(cfg, stokes="mixed")
        for _ in range(4):                  # the recorded ensemble ran one eager step first
            m.step()
        assert d["stokes"]["converged"] == 1
        for xa, xb in zip(st, _state(m)):
            assert np.array_equal(xa, xb), cfg.name


def test_recorded_step_with_idle_learned_guess():
    """The learned guess is consulted at cold starts only; while it is idle the recorded step
    stands in for the step with the hook, and a reset (cold start) runs eagerly with the hook."""
    import os
    from meeuuw_b200 import configs
    from meeuuw_b200.timestep import GPUModel
    from meeuuw_b200.unet import LearnedGuess, UNet
    weights = os.path.join(os.path.dirname(os.path.dirname(__file__)), "meeuuw_b200", "weights", "unet_fk128.npz")
    net = UNet.load(weights)
    cfg = configs.fk_convection(32, seed=7, Ra=1e5)
    host = configs.build_host_model(cfg)
    a = GPUModel(cfg, host, stokes="mixed")
    b = GPUModel(cfg, host, stokes="mixed")
    a.guess, b.guess = LearnedGuess(a, net), LearnedGuess(b, net)
    for _ in range(4):
        a.step()
    b.step()                                # the cold start consults the network
    assert b.guess.idle()
    b.capture_step()
    for _ in range(3):
        b.step()
    assert b._replayed
    for xa, xb in zip(_state(a), _state(b)):
        assert np.array_equal(xa, xb)
    assert a.guess.picks == b.guess.picks
    a.guess.reset()
    b.guess.reset()
    a.step()
    b.step()                                # cold again: eager, with the hook
    assert not b._replayed and b.guess.idle()
    a.step()
    b.step()                                # idle: the recorded step again
    assert b._replayed
    da, db = a.diagnostics(), b.diagnostics()
    for xa, xb in zip(_state(a), _state(b)):
        assert np.array_equal(xa, xb)
    assert a.guess.picks == b.guess.picks and da["vrms"] == db["vrms"]
