"""The ensemble's Stokes solves in one launch (one thread-block cluster per model) against each
model's own solver.

* Solve level: models of uneven size (partial element tiles, dense and smoothed coarsest levels,
  two to five multigrid levels) solved from the same right-hand sides, viscosities and guesses by
  the per-model mixed solver and by the cluster solve.  Both must reach the FP64 relative
  residual 1e-8 (checked independently with mw_stokes_residual) with outer iteration counts
  within 2 of each other; the solutions agree to 1e-6 relative (two solutions each within the
  tolerance; the dot products are summed in another order).
* Step level: three steps of a BatchedEnsemble (each model's phases before and after the solve
  replayed from its own recorded graphs; with a size limit, the larger models' whole steps) against
  the same models stepped alone: vrms and Nu within 1e-6 relative, positions within 1e-9.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _models(ns, seed=5):
    from meeuuw_b200.ensemble import sample_configs
    from meeuuw_b200.timestep import GPUModel
    from dataclasses import replace
    from meeuuw_b200 import configs
    out = []
    for i, n in enumerate(ns):
        cfg = replace(configs.fk_convection(n), name=f"b{i}_{n}", fk_gamma=np.log(10.0 ** (1 + i)), seed=seed + i)
        out.append(GPUModel(cfg, stokes="mixed"))
    return out


@pytest.mark.parametrize("ns", [(40, 24, 64, 18), (96, 30)])
def test_cluster_solve_matches_per_model_solver(ns):
    from meeuuw_b200 import ops
    from meeuuw_b200.stokes import StokesEnsembleSolve
    models = _models(ns)
    for m in models:
        with ops.workspace_scope(m):
            m._step_pre()
    guesses = [(m.solV.clone(), m.solP.clone()) for m in models]
    ref = []
    for m in models:
        V, P, info = m.solver.solve(m.rhs_f, m.rhs_h, m.solV, m.solP, **m.stokes_solve_kw())
        assert info["converged"] == 1, info
        ref.append((V.clone(), P.clone(), info))
    for m, (V0, P0) in zip(models, guesses):
        m.solV.copy_(V0)
        m.solP.copy_(P0)
        m.solver.prepare("mixed")
    ens = StokesEnsembleSolve([m.solver for m in models], [m.rhs_f for m in models], [m.rhs_h for m in models],
                              [m.solV for m in models], [m.solP for m in models])
    kw = models[0].stokes_solve_kw()
    kw.pop("precision")
    ens.solve(use_guess=True, **kw)
    torch.cuda.synchronize()
    for m, (Vr, Pr, ir) in zip(models, ref):
        info = m.solver.device_info(m.tol)
        assert info["converged"] == 1 and info["rel_residual"] <= m.tol, (m.cfg.name, info)
        _, _, nrm = m.solver.residual(m.solV, m.solP, m.rhs_f, m.rhs_h)
        bn = float(torch.sqrt((m.rhs_f ** 2).sum() + (m.rhs_h ** 2).sum()))
        assert nrm / bn <= 1.001 * m.tol, (m.cfg.name, nrm / bn)
        assert abs(info["outer_iters"] - ir["outer_iters"]) <= 2, (m.cfg.name, info, ir)
        assert info["refinements"] >= 1
        dv = float((m.solV - Vr).norm() / Vr.norm())
        assert dv < 1e-6, (m.cfg.name, dv)


@pytest.mark.parametrize("cluster_max_nel", [None, 900])
def test_batched_ensemble_steps_match_models_alone(cluster_max_nel):
    """cluster_max_nel=900: the larger models step alone (whole-step graphs) beside the cluster solve."""
    from meeuuw_b200.ensemble import BatchedEnsemble, sample_configs
    from meeuuw_b200.timestep import GPUModel
    cfgs = sample_configs(4, seed=3, n_range=(16, 48), Ra_range=(1e4, 1e6), contrast_range=(1.0, 1e3))
    ens = BatchedEnsemble(cfgs, cluster_max_nel=cluster_max_nel)
    if cluster_max_nel is not None:
        assert ens.batched and ens.alone, [c.nel for c in cfgs]
    for _ in range(3):
        ens.step()
    ens.synchronize()
    ens.check()
    got = ens.diagnostics()
    xs = [m.x.cpu().numpy() for m in ens.models]
    assert len(ens.graphs) == len(cfgs) and not ens.retired
    for cfg, d, x in zip(cfgs, got, xs):
        assert d["istep"] == 4 and d["stokes"]["converged"] == 1, (cfg.name, d)
        m = GPUModel(cfg, stokes="mixed")
        for _ in range(4):
            m.step()
        r = m.diagnostics()
        assert abs(d["vrms"] / r["vrms"] - 1) < 1e-6, (cfg.name, d["vrms"], r["vrms"])
        assert abs(d["Nu"] / r["Nu"] - 1) < 1e-6, (cfg.name, d["Nu"], r["Nu"])
        assert np.max(np.abs(x - m.x.cpu().numpy())) < 1e-9, cfg.name


def test_mode_tuner_on_device(tmp_path):
    """The strategy tuner builds and times real ensembles and returns a working one."""
    from meeuuw_b200.ensemble import ModeTuner, default_modes, sample_configs
    cfgs = sample_configs(3, seed=5, n_range=(16, 32), Ra_range=(1e4, 1e5), contrast_range=(1.0, 1e2))
    modes = {k: v for k, v in default_modes().items() if k in ("graphs", "batched")}
    name, ens, t = ModeTuner(cache_path=str(tmp_path / "m.json"), modes=modes).tune(cfgs, steps=1)
    assert name in modes and set(t) == set(modes) and min(t.values()) == t[name]
    ens.step()
    ens.synchronize()
    ens.check()
    assert all(d["stokes"]["converged"] == 1 for d in ens.diagnostics())
