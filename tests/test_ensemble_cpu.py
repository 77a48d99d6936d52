"""Host-side logic of the ensemble layer (no GPU): the uneven ensemble's sampling and the
autotuner's choice and cache."""
import math
import time

import torch

from meeuuw_b200.ensemble import Autotuner, sample_configs


def test_sample_configs_ranges_and_seeds():
    cfgs = sample_configs(64, seed=3)
    assert len(cfgs) == 64
    ns = [c.nelx for c in cfgs]
    assert all(64 <= n <= 192 and n % 2 == 0 and c.nelz == n for n, c in zip(ns, cfgs))
    assert len(set(ns)) > 10                                 # uneven sizes
    assert all(1e4 <= c.Ra <= 1e7 for c in cfgs)
    assert all(0.0 <= c.fk_gamma <= math.log(1e4) + 1e-12 for c in cfgs)
    assert all(c.nparticle_per_dim == 4 for c in cfgs)
    assert len({c.seed for c in cfgs}) == 64
    assert [c.nelx for c in sample_configs(64, seed=3)] == ns   # reproducible


class _FakeModel:
    def __init__(self, nel):
        self.nel = nel


class _FakeEnsemble:
    """Step time falls until 4 threads, then rises: the tuner must pick 4."""

    def __init__(self):
        self.models = [_FakeModel(4096 * (i + 1)) for i in range(8)]
        self.threads = 1

    def set_threads(self, t):
        self.threads = t

    def step(self):
        time.sleep(0.004 * abs(math.log2(self.threads) - 2) + 0.002)

    def synchronize(self):
        pass


def test_autotuner_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a: "fake-gpu")
    path = tmp_path / "tune.json"
    ens = _FakeEnsemble()
    rec = Autotuner(cache_path=str(path), candidates=(1, 2, 4, 8, 16)).tune(ens, steps=2)
    assert rec["threads"] == 4 and ens.threads == 4
    assert 16 not in rec["seconds_per_step"]                 # more threads than models are skipped
    ens2 = _FakeEnsemble()
    rec2 = Autotuner(cache_path=str(path)).tune(ens2)
    assert rec2["threads"] == 4 and ens2.threads == 4        # from the cache, without timing


class _FakeModeEnsemble:
    """An ensemble whose step takes `dt` seconds."""

    def __init__(self, dt):
        self.dt, self.closed = dt, False

    def step(self):
        time.sleep(self.dt)

    def synchronize(self):
        pass

    def close(self):
        self.closed = True


def test_mode_tuner_picks_fastest_strategy_and_caches(tmp_path, monkeypatch):
    from meeuuw_b200.ensemble import ModeTuner
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a: "fake-gpu")
    built = []

    def mode(dt):
        def build(cfgs):
            e = _FakeModeEnsemble(dt)
            built.append(e)
            return e
        return build
    modes = {"graphs": mode(0.004), "threads": mode(0.012), "batched": mode(0.020)}
    cfgs = sample_configs(4, seed=1)
    path = tmp_path / "modes.json"
    name, ens, t = ModeTuner(cache_path=str(path), modes=modes).tune(cfgs, steps=2)
    assert name == "graphs" and ens is built[0] and set(t) == set(modes)
    assert t["graphs"] < t["threads"] < t["batched"]
    assert not built[0].closed and built[1].closed and built[2].closed   # the others released
    built.clear()
    name2, ens2, _ = ModeTuner(cache_path=str(path), modes=modes).tune(cfgs)
    assert name2 == "graphs" and len(built) == 1                        # from the cache: one build
