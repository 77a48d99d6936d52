"""Ensembles of independent models of uneven size advanced together on one GPU.

A small model (64² elements: 4096 elements, 65 k particles) fills a fraction of a B200: its
operator applies launch 32 thread blocks on 148 SMs, and its host-side launch sequence leaves the
GPU idle between kernels.  An ensemble therefore runs every model on its own CUDA stream and
advances the models concurrently from a pool of host threads (the C ABI calls release the
interpreter lock, so launches from different threads overlap), letting the GPU interleave the
models' kernels.  Each model keeps its own device buffers, scratch (per-stream workspaces) and
Stokes solver (its own stream and recorded CUDA graphs), so nothing is shared between models.

``Autotuner`` picks the number of host threads (the concurrency level) by timing ensemble steps,
and caches the choice per GPU and ensemble shape.

``BatchedEnsemble`` runs the Stokes solves of the models in one launch instead (one thread-block
cluster per model running that model's whole mixed-precision solve,
``stokes.StokesEnsembleSolve``), between the models' other phases, which replay from recorded
graphs on the models' own streams.

Many streams share the GPU's hardware work queues (CUDA_DEVICE_MAX_CONNECTIONS, 8 by default): a
process running a large ensemble should set it higher (up to 32) before CUDA is initialised, so
that one model's device-side solver loop does not hold up the models queued behind it.
"""
import json
import math
import os
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import replace

import numpy as np
import torch

from . import configs, ops
from .stokes import StokesEnsembleSolve
from .timestep import GPUModel


def sample_configs(n_models=64, seed=0, n_range=(64, 192), Ra_range=(1e4, 1e7), contrast_range=(1.0, 1e4),
                   nparticle_per_dim=4):
    """Uneven ensemble: square grids n ~ U[n_range] (even), Ra and the Frank-Kamenetskii viscosity
    contrast log-uniform, 16 particles per element, a seed per model."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_models):
        n = int(rng.integers(n_range[0] // 2, n_range[1] // 2 + 1)) * 2
        Ra = math.exp(rng.uniform(math.log(Ra_range[0]), math.log(Ra_range[1])))
        c = math.exp(rng.uniform(math.log(contrast_range[0]), math.log(contrast_range[1])))
        base = configs.fk_convection(n)
        out.append(replace(base, name=f"ens{i}_{n}", Ra=Ra, fk_gamma=math.log(c), seed=int(seed * 100003 + i),
                           nparticle_per_dim=nparticle_per_dim))
    return out


class Ensemble:
    """N independent models, each on its own stream, stepped concurrently by `threads` host threads.

    CUDA maps streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware work queues (8 unless the
    environment says otherwise when CUDA initialises); with more models than queues, streams share
    queues and their launches serialise.  Set it to 32 before the first CUDA call (bench.py
    --ensemble does): 88 -> 129 model-steps/s for 64 models (measured)."""

    def __init__(self, cfgs, stokes="mixed", threads=8, tol=1e-8, guess=None, graphs=False):
        """graphs=True records each model's whole time step as one CUDA graph (after one eager
        step); a step of the ensemble is then one graph launch per model, issued from one thread.
        guess: a factory model -> Stokes guess hook (e.g. unet.LearnedGuess, consulted at the cold
        start); with graphs the cold first step runs eagerly with the hook, then the step is
        recorded (the hook is idle from then on).  first_step_info holds each model's first-step
        solver statistics when that step ran here."""
        self.cfgs = list(cfgs)
        self.streams, self.models = [], []
        self.graphs = bool(graphs)
        self.first_step_info = []
        for cfg in self.cfgs:
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                m = GPUModel(cfg, stokes=stokes, tol=tol)
                if guess is not None:
                    m.guess = guess(m)
                if self.graphs:
                    m.step()                      # the cold start (with the hook, if any)
                    self.first_step_info.append(dict(m.last_solve))
                    m.capture_step()
            self.streams.append(st)
            self.models.append(m)
        torch.cuda.synchronize()
        if self.graphs:
            self.steps_done = len(self.models)
        self.active = [True] * len(self.models)
        self.retired = {}            # model index -> the reference's abort message
        if not self.graphs:
            self.steps_done = 0      # model-steps taken by active models
        self.threads = 0
        self.pool = None
        self.set_threads(threads)

    def set_threads(self, threads):
        threads = max(1, min(int(threads), len(self.models)))
        if threads != self.threads:
            if self.pool is not None:
                self.pool.shutdown(wait=True)
            self.pool = ThreadPoolExecutor(max_workers=threads)
            self.threads = threads

    def _run(self, idx):
        done = 0
        for i in idx:
            with torch.cuda.stream(self.streams[i]):
                m = self.models[i]
                m.step()
                done += 1
                if int(m.err.item()):
                    # the reference would abort this run (an empty element, a particle outside
                    # the box): retire the model, keep the others going
                    try:
                        m.check()
                        self.retired[i] = f"device flags {int(m.err.item())}"
                    except SystemExit as e:
                        self.retired[i] = str(e)
                    self.active[i] = False
        return done

    def _retire_flagged(self, idx):
        for i in idx:
            m = self.models[i]
            with torch.cuda.stream(self.streams[i]):
                flags = int(m.err.item())
            if flags:
                try:
                    m.check()
                    self.retired[i] = f"device flags {flags}"
                except SystemExit as e:
                    self.retired[i] = str(e)
                self.active[i] = False

    def step(self):
        """One time step of every active model.  Recorded steps: every model's graph is launched on
        its stream, then the flags are read.  Otherwise models are dealt to the threads largest
        first, so each thread gets a similar amount of work."""
        if self.graphs:
            idx = sorted((i for i in range(len(self.models)) if self.active[i]), key=lambda i: -self.models[i].nel)
            for i in idx:
                with torch.cuda.stream(self.streams[i]):
                    self.models[i].step()
            self.steps_done += len(idx)
            self._retire_flagged(idx)
            return
        order = sorted((i for i in range(len(self.models)) if self.active[i]), key=lambda i: -self.models[i].nel)
        parts = [order[t::self.threads] for t in range(self.threads)]
        futs = [self.pool.submit(self._run, p) for p in parts if p]
        for f in futs:
            self.steps_done += f.result()

    def synchronize(self):
        for st in self.streams:
            st.synchronize()

    def diagnostics(self):
        return [m.diagnostics() for m in self.models]

    def check(self):
        """SystemExit when any model still stepping has a device flag set."""
        for i, m in enumerate(self.models):
            if self.active[i]:
                m.check()

    def close(self):
        if self.pool is not None:
            self.pool.shutdown(wait=True)
            self.pool = None


class BatchedEnsemble:
    """N independent models whose Stokes solves run in one launch.

    A step: every model's phases up to the solve (particles, projections, right-hand side,
    viscosity, multigrid hierarchy) replayed from the model's own recorded graph on its own stream;
    then one launch in which a thread-block cluster per model runs that model's whole solve (its
    own hierarchy, iteration counts and convergence tests, no waiting between clusters); then every
    model's phases after the solve (energy, Nu, vrms, advection, locate), again one recorded graph
    per model on its stream.  Models with more than `cluster_max_nel` elements (None: no limit)
    instead replay their whole step as one graph on their own stream, concurrently, since one
    cluster (8 CTAs) works through a large model's solve more slowly than the whole GPU does.
    Every model's cold first step runs eagerly (with the guess hook, if one is given).  A model
    whose device flags are set is retired with the reference's message."""

    def __init__(self, cfgs, tol=1e-8, guess=None, cluster_max_nel=None):
        self.cfgs = list(cfgs)
        self.models, self.streams = [], []
        self.first_step_info = []
        for cfg in self.cfgs:
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                m = GPUModel(cfg, stokes="mixed", tol=tol)
                if guess is not None:
                    m.guess = guess(m)
                m.step()                          # the cold start: per-model solve (and hook)
                self.first_step_info.append(dict(m.last_solve))
                if m.guess is not None and not m._guess_idle():
                    raise ValueError("the guess hook must be idle after the first step")
            self.models.append(m)
            self.streams.append(st)
        torch.cuda.synchronize()
        self.active = [True] * len(self.models)
        self.retired = {}
        self.steps_done = len(self.models)
        self.cluster_max_nel = cluster_max_nel
        self.main = torch.cuda.Stream()
        self.graphs = {}                          # model index -> (pre, post) or whole-step graph
        self._bind()

    def _in_cluster(self, i):
        return self.cluster_max_nel is None or self.models[i].nel <= self.cluster_max_nel

    def _bind(self):
        self.idx = [i for i in range(len(self.models)) if self.active[i]]
        self.batched = [i for i in self.idx if self._in_cluster(i)]
        self.alone = [i for i in self.idx if not self._in_cluster(i)]
        ms = [self.models[i] for i in self.batched]
        self.solve = StokesEnsembleSolve([m.solver for m in ms], [m.rhs_f for m in ms], [m.rhs_h for m in ms],
                                         [m.solV for m in ms], [m.solP for m in ms]) if ms else None

    def _record(self, i):
        """The model's recorded graphs: (pre, post) around the shared solve, or its whole step."""
        if i in self.graphs:
            return self.graphs[i]
        m, st = self.models[i], self.streams[i]
        torch.cuda.synchronize()
        if not self._in_cluster(i):
            with torch.cuda.stream(st):
                m.capture_step()
            self.graphs[i] = m.graph
            return m.graph
        gs = []
        for body in (lambda: (m._step_pre(), m.solver.prepare("mixed")), m._step_post):
            g = torch.cuda.CUDAGraph()
            m._capturing = True
            try:
                with torch.cuda.stream(st), ops.workspace_scope(m):
                    with torch.cuda.graph(g, stream=st, capture_error_mode="thread_local"):
                        body()
            finally:
                m._capturing = False
            gs.append(g)
        m.istep -= 1                              # the post capture counted a step; nothing ran
        self.graphs[i] = tuple(gs)
        return self.graphs[i]

    def step(self):
        """One time step of every active model."""
        if not self.idx:
            return
        rec = {i: self._record(i) for i in self.idx}
        main = self.main
        main.wait_stream(torch.cuda.current_stream())
        for i in self.alone:                      # whole steps, concurrently with the rest
            st = self.streams[i]
            st.wait_stream(main)
            with torch.cuda.stream(st):
                self.models[i].step()
        for i in self.batched:                    # fork every model from main first, ...
            self.streams[i].wait_stream(main)
        for i in self.batched:
            with torch.cuda.stream(self.streams[i]):
                rec[i][0].replay()
        for i in self.batched:                    # ... then join them all (a join inside the fork
            main.wait_stream(self.streams[i])     # loop would chain the models one after another)
        if self.batched:
            m0 = self.models[self.batched[0]]
            kw = m0.stokes_solve_kw()
            kw.pop("precision")
            with torch.cuda.stream(main):
                self.solve.solve(use_guess=True, **kw)
        for i in self.batched:
            self.streams[i].wait_stream(main)
        for i in self.batched:
            with torch.cuda.stream(self.streams[i]):
                rec[i][1].replay()
            m = self.models[i]
            m._replayed = True                    # outcomes are on the device
            m.istep += 1
        cur = torch.cuda.current_stream()
        for i in self.idx:
            cur.wait_stream(self.streams[i])
        self.steps_done += len(self.idx)
        self._retire_flagged()

    def _retire_flagged(self):
        changed = False
        for i in self.idx:
            m = self.models[i]
            with torch.cuda.stream(self.streams[i]):
                flags = int(m.err.item())
            if flags:
                try:
                    m.check()
                    self.retired[i] = f"device flags {flags}"
                except SystemExit as e:
                    self.retired[i] = str(e)
                self.active[i] = False
                changed = True
        if changed:
            self._bind()

    def synchronize(self):
        torch.cuda.synchronize()

    def diagnostics(self):
        return [m.diagnostics() for m in self.models]

    def check(self):
        for i, m in enumerate(self.models):
            if self.active[i]:
                m.check()


class Autotuner:
    """Picks an ensemble's concurrency level (host threads) by timing a few steps at each candidate,
    keeping the fastest; the choice is cached in a JSON file keyed by GPU name and the ensemble's
    element counts."""

    def __init__(self, cache_path=None, candidates=(1, 2, 4, 8, 16, 32)):
        self.cache_path = cache_path or os.path.join(os.path.expanduser("~"), ".cache", "meeuuw_b200_autotune.json")
        self.candidates = candidates

    def _key(self, ens):
        name = torch.cuda.get_device_name()
        sizes = sorted(m.nel for m in ens.models)
        return f"{name}|{len(sizes)}|{sum(sizes)}|{sizes[0]}|{sizes[-1]}"

    def _load(self):
        try:
            with open(self.cache_path) as f:
                return json.load(f)
        except Exception:
            return {}

    def tune(self, ens, steps=2, use_cache=True):
        key = self._key(ens)
        cache = self._load()
        if use_cache and key in cache:
            ens.set_threads(cache[key]["threads"])
            return cache[key]
        timings = {}
        for t in self.candidates:
            if t > len(ens.models):
                continue
            ens.set_threads(t)
            ens.step()                     # settle (graph recording, workspaces) at this level
            ens.synchronize()
            t0 = time.perf_counter()
            for _ in range(steps):
                ens.step()
            ens.synchronize()
            timings[t] = (time.perf_counter() - t0) / steps
        best = min(timings, key=timings.get)
        ens.set_threads(best)
        rec = {"threads": best, "seconds_per_step": timings}
        cache[key] = {"threads": best, "seconds_per_step": {str(k): v for k, v in timings.items()}}
        try:
            os.makedirs(os.path.dirname(self.cache_path), exist_ok=True)
            with open(self.cache_path, "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
        return rec


def default_modes(guess=None, tol=1e-8):
    """The ensemble's execution strategies, by name: builders cfgs -> ensemble."""
    return {
        "graphs": lambda cfgs: Ensemble(cfgs, stokes="mixed", tol=tol, graphs=True, guess=guess),
        "threads": lambda cfgs: Ensemble(cfgs, stokes="mixed", tol=tol, threads=32, guess=guess),
        "batched": lambda cfgs: BatchedEnsemble(cfgs, tol=tol, guess=guess),
        "batched_le6000": lambda cfgs: BatchedEnsemble(cfgs, tol=tol, guess=guess, cluster_max_nel=6000),
    }


class ModeTuner:
    """Picks an ensemble's execution strategy -- one recorded step per model, the thread pool, every
    Stokes solve in one cluster launch, or that launch for the smaller models only -- by building
    each candidate on the given models and timing a few steps after one settling step; the fastest
    is kept (its ensemble is returned, the others released).  The choice is cached in a JSON file
    keyed by GPU name and the ensemble's element counts, so later runs build only the chosen one.
    Timing with several candidates changes nothing but the state of the returned ensemble's models,
    which have taken the settling and timed steps."""

    def __init__(self, cache_path=None, modes=None):
        self.cache_path = cache_path or os.path.join(os.path.expanduser("~"), ".cache", "meeuuw_b200_modes.json")
        self.modes = modes if modes is not None else default_modes()

    @staticmethod
    def _key(cfgs):
        name = torch.cuda.get_device_name()
        sizes = sorted(c.nel for c in cfgs)
        return f"{name}|{len(sizes)}|{sum(sizes)}|{sizes[0]}|{sizes[-1]}"

    def _load(self):
        try:
            with open(self.cache_path) as f:
                return json.load(f)
        except Exception:
            return {}

    def tune(self, cfgs, steps=2, use_cache=True):
        """(mode name, its ensemble, seconds per step of every candidate timed)."""
        key = self._key(cfgs)
        cache = self._load()
        if use_cache and key in cache and cache[key]["mode"] in self.modes:
            name = cache[key]["mode"]
            return name, self.modes[name](cfgs), cache[key]["seconds_per_step"]
        timings, best, best_ens = {}, None, None
        for name, build in self.modes.items():
            ens = build(cfgs)
            ens.step()                            # settle: recording, workspaces
            ens.synchronize()
            t0 = time.perf_counter()
            for _ in range(steps):
                ens.step()
            ens.synchronize()
            timings[name] = (time.perf_counter() - t0) / steps
            if best is None or timings[name] < timings[best]:
                if best_ens is not None and hasattr(best_ens, "close"):
                    best_ens.close()
                best, best_ens = name, ens
            elif hasattr(ens, "close"):
                ens.close()
        cache[key] = {"mode": best, "seconds_per_step": timings}
        try:
            os.makedirs(os.path.dirname(self.cache_path), exist_ok=True)
            with open(self.cache_path, "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
        return best, best_ens, timings
