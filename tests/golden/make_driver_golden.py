"""Whole-run fixtures from the reference's own driver, ``meeuuw.py``.

Run in a container that holds the reference checkout (read from ``/root/reference``;
nothing at test time reads it):

    python tests/golden/make_driver_golden.py [case ...]

Each case runs the unmodified driver (``runpy`` on ``meeuuw.py``) with its own
command-line options, in a scratch directory that receives the driver's output files.
Two things are supplied from outside the checkout:

* a permissive ``matplotlib`` stub (the PNG writers import it; this image has none);
* a shadow ``experiment<e>`` module that executes the reference's experiment module and
  then switches its mesh stretching off, so ``--nelx/--nelz`` give the uniform box
  (experiment 0 stretches with fixed segment counts, ``experiment0.py:53-62``, which
  breaks resolution overrides), and optionally replaces globals (noted per case; the
  output frequencies only change which files the driver writes).

Per time step the reference's own calls are recorded by wrapping the functions the
driver star-imports (``meeuuw.py:14-72``) before it runs: vrms from
``compute_global_quantities`` (``meeuuw.py:2512``), Nu from ``compute_Nu``
(``meeuuw.py:2298``), dt from the ``advect_particles___box`` call (``meeuuw.py:2726``).
The final state (T, u, w, p, q, strain rate, swarm) comes from the driver's globals;
large meshes keep a subsample (listed in ``nodes``, ``pnodes``, ``particles``) and the
per-element particle counts.  Particles are placed regularly (``particle_distribution=1``),
so no random draw is involved.
"""
import json
import os
import runpy
import sys
import tempfile
import types

import numpy as np

REF = "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))

# output frequencies only: the writers do not touch the computed state
_QUIET = {k: 10 ** 9 for k in ("every_solution", "every_solution_vtu", "every_solution_png", "every_swarm_vtu",
                                "every_swarm_png", "every_swarm_ascii", "every_quadpoints_vtu")}

# name -> (experiment, nel, nstep, extra argv, globals replaced after the experiment module)
CASES = {
    # config 0: Blankenbach 1a (Ra 1e4, isoviscous), 32x32, 4x4 regular particles, RK2, CN, direct solve
    "driver_c0_32": (0, 32, 20, ["--RKorder", "2", "--particle_distribution", "1",
                                 "--nparticle_per_dim", "4"], {}),
    # the same at 16x16 for 3 steps, with a temperature-dependent viscosity (experiment 0's case 2a
    # law, eta = exp(-6.907755279 T), elemental geometric averaging) so the material path is pinned too
    "driver_fk_16": (0, 16, 3, ["--RKorder", "4", "--particle_distribution", "1",
                                "--nparticle_per_dim", "4", "--averaging", "2"], {"icase": "2a"}),
    # config 2's set-up as the reference ships it (experiment1.py: 0.9142 x 1 box, interface
    # z = 0.2 + 0.02 cos(pi x / 0.9142), rho 1000 below / 1010 above, no slip top and bottom,
    # volume pressure normalisation), 25 regular particles per element, RK2
    "driver_rt_64": (1, 64, 20, ["--particle_distribution", "1", "--nparticle_per_dim", "5"], _QUIET),
    "driver_rt_256": (1, 256, 2, ["--particle_distribution", "1", "--nparticle_per_dim", "5"], _QUIET),
}


class _Any:
    """Accepts every attribute access and call (the PNG writers' matplotlib use)."""

    def __getattr__(self, k):
        return _Any()

    def __call__(self, *a, **k):
        return _Any()


def _stub_matplotlib():
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.__getattr__ = lambda k: _Any()
    plt.__getattr__ = lambda k: _Any()
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt


def _shadow_experiment(tmp, e, overrides):
    """A module ``experiment<e>`` placed ahead of the checkout on sys.path."""
    src = (
        "import importlib.util as _u\n"
        f"_s = _u.spec_from_file_location('_ref_experiment{e}', {os.path.join(REF, f'experiment{e}.py')!r})\n"
        "_m = _u.module_from_spec(_s)\n"
        "_s.loader.exec_module(_m)\n"
        "for _k, _v in vars(_m).items():\n"
        "    if not _k.startswith('__'):\n"
        "        globals()[_k] = _v\n"
        "use_stretching_x = False\n"
        "use_stretching_z = False\n"
    )
    for k, v in overrides.items():
        src += f"{k} = {v!r}\n_m.{k} = {v!r}\n"
    d = os.path.join(tmp, "shadow")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, f"experiment{e}.py"), "w") as f:
        f.write(src)
    return d


def run_case(name):
    e, n, nstep, argv, overrides = CASES[name]
    saved_path, saved_argv, saved_cwd = list(sys.path), list(sys.argv), os.getcwd()
    rec = {"vrms": [], "Nu": [], "dt": [], "Tavrg": []}
    with tempfile.TemporaryDirectory() as tmp:
        shadow = _shadow_experiment(tmp, e, overrides)
        _stub_matplotlib()
        for k in list(sys.modules):
            if k.startswith("experiment"):
                del sys.modules[k]
        sys.path[:0] = [shadow, REF]
        import pic_functions
        import postprocessors

        gq, nu, adv = (postprocessors.compute_global_quantities, postprocessors.compute_Nu,
                       pic_functions.advect_particles___box)

        def gq_rec(*a, **k):
            out = gq(*a, **k)
            rec["vrms"].append(float(out[0]))
            rec["Tavrg"].append(float(out[7]))
            return out

        def nu_rec(*a, **k):
            out = nu(*a, **k)
            rec["Nu"].append(float(out[-1]))
            return out

        def adv_rec(RKorder, dt, *a, **k):
            rec["dt"].append(float(dt))
            return adv(RKorder, dt, *a, **k)

        postprocessors.compute_global_quantities = gq_rec
        postprocessors.compute_Nu = nu_rec
        pic_functions.advect_particles___box = adv_rec
        try:
            os.chdir(tmp)
            sys.argv = ["meeuuw.py", "--e", str(e), "--nelx", str(n), "--nelz", str(n), "--nstep", str(nstep),
                        "--output_folder", os.path.join(tmp, "OUT")] + argv
            g = runpy.run_path(os.path.join(REF, "meeuuw.py"), run_name="__main__")
        finally:
            os.chdir(saved_cwd)
            sys.path[:] = saved_path
            sys.argv = saved_argv
            postprocessors.compute_global_quantities = gq
            postprocessors.compute_Nu = nu
            pic_functions.advect_particles___box = adv
    out = {k: np.asarray(v, dtype=np.float64) for k, v in rec.items()}
    nn_V, nel = int(g["nn_V"]), int(g["nel"])
    nodes = np.arange(nn_V)
    if nn_V > 20000:            # large meshes: every fourth node of every fourth node row
        nnx = 2 * n + 1
        nodes = nodes[((nodes % nnx) % 4 == 0) & ((nodes // nnx) % 4 == 0)]
    out["nodes"] = nodes.astype(np.int32)
    fields = ("u", "w", "q") + (("T",) if bool(g["solve_T"]) else ())
    if nn_V <= 5000:
        fields += ("exx_n", "ezz_n", "exz_n")
    for k in fields:
        out[k] = np.asarray(g[k], dtype=np.float64)[nodes]
    pnodes = np.arange(int(g["nn_P"]))
    if nn_V > 20000:            # the pressure nodes that coincide with the velocity nodes kept
        pnodes = pnodes[((pnodes % (n + 1)) % 2 == 0) & ((pnodes // (n + 1)) % 2 == 0)]
    out["pnodes"] = pnodes.astype(np.int32)
    out["p"] = np.asarray(g["p"], dtype=np.float64)[pnodes]
    act = np.asarray(g["swarm_active"], dtype=bool)
    iel = np.asarray(g["swarm_iel"], dtype=np.int32)
    out["counts"] = np.bincount(iel[act], minlength=nel).astype(np.int32)
    npart = len(act)
    parts = np.arange(0, npart, max(1, npart // 16384))
    out["particles"] = parts.astype(np.int32)
    out["swarm_x"] = np.asarray(g["swarm_x"], dtype=np.float64)[parts]
    out["swarm_z"] = np.asarray(g["swarm_z"], dtype=np.float64)[parts]
    out["swarm_active"] = act[parts]
    out["swarm_iel"] = iel[parts]
    if "swarm_wf" in g and int(g["nmat"]) > 1:          # material id = the material of weight 1
        out["swarm_mat"] = np.argmax(np.asarray(g["swarm_wf"]), axis=0).astype(np.int8)[parts]
    meta = dict(experiment=e, nel=n, nstep=nstep, Ra=float(g.get("Ra", float("nan"))), RKorder=int(g["RKorder"]),
                averaging=str(g["averaging"]), nparticle_per_dim=int(g["nparticle_per_dim"]),
                CFLnb=float(g["CFLnb"]), solve_T=bool(g["solve_T"]),
                pressure_normalisation=str(g["pressure_normalisation"]), argv=" ".join(argv),
                overrides=repr({k: v for k, v in overrides.items() if k not in _QUIET}))
    out["meta"] = np.array(json.dumps(meta))
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(name, {k: (v.shape if v.ndim else v) for k, v in out.items()}, "->", path)


if __name__ == "__main__":
    for c in (sys.argv[1:] or list(CASES)):
        run_case(c)
