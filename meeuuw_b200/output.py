"""Solution and swarm output (VTU, ASCII, PVD collections) streamed from device buffers.

The reference writes its output from host arrays inside the time loop
(``output_solution_to_vtu.py:12-436``, ``output_swarm_to_vtu.py:12-212``,
``output_swarm_to_ascii.py:12-107``, ``write_in_pvd_files.py:8-39``; called at
``meeuuw.py:1984-2058``, ``:3043-3110``, ``:3164``), so every output step waits for the files.
Here a step's fields are first copied device to device into a snapshot slot on the model's
stream (a few hundred microseconds at 512x512), then copied to pinned host memory on a side
stream and written by a background thread: the next time step runs while the previous one's
files are formatted.  Two snapshot slots alternate; a third output request waits only for the
older slot's copy, never for a file.

The files follow the reference's layout: the same XML skeleton, array names and number formats
(ASCII), biquadratic cells (VTK type 28) with the reference's node order, one vertex cell per
active particle, and ``solution.pvd`` / ``swarm.pvd`` collections whose entries name
``solution_%04d.vtu`` and ``SWARM/swarm_%04d.vtu``.
"""
import os
import queue
import threading

import numpy as np
import torch


# ---------------------------------------------------------------------------------------- writers
def q2_connectivity(nelx, nelz):
    """(9, nel) node indices in the reference's order (build_velocity_connectivity.py:63-92)."""
    nnx = 2 * nelx + 1
    ez, ex = np.meshgrid(np.arange(nelz), np.arange(nelx), indexing="ij")
    b = (ex * 2 + ez * 2 * nnx).ravel()
    return np.stack([b, b + 2, b + 2 + 2 * nnx, b + 2 * nnx, b + 1, b + 2 + nnx,
                     b + 1 + 2 * nnx, b + nnx, b + 1 + nnx]).astype(np.int64)


def _array(f, name, data, fmt, ncomp=1, kind="Float32"):
    comp = f" NumberOfComponents='{ncomp}'" if ncomp > 1 else ""
    nm = f" Name='{name}'" if name else ""
    f.write(f"<DataArray type='{kind}'{comp}{nm} Format='ascii'> \n")
    if ncomp > 1:
        np.savetxt(f, data, fmt=fmt)
    else:
        np.asarray(data).tofile(f, sep=" ", format=fmt)
    f.write("</DataArray>\n")


def write_solution_vtu(path, nelx, nelz, x_V, z_V, nodal, elemental):
    """output_solution_to_vtu.py:87-436 for the fields given.  nodal: {name: (nn_V,) or
    ("vector", u, w)}; elemental: {name: (nel,)} (integer arrays are written as Int32)."""
    nn, nel = len(x_V), nelx * nelz
    icon = q2_connectivity(nelx, nelz)
    with open(path, "w") as f:
        f.write("<VTKFile type='UnstructuredGrid' version='0.1' byte_order='BigEndian'> \n")
        f.write("<UnstructuredGrid> \n")
        f.write("<Piece NumberOfPoints=' %5d ' NumberOfCells=' %5d '> \n" % (nn, nel))
        f.write("<Points> \n")
        _array(f, None, np.stack([x_V, np.zeros(nn), z_V], axis=1), "%.5e %.1e %.5e", 3)       # :91-96
        f.write("</Points> \n")
        f.write("<PointData Scalars='scalars'>\n")
        for name, v in nodal.items():
            if isinstance(v, tuple):                                                        # :100-105
                _array(f, name, np.stack([v[1], np.zeros(nn), v[2]], axis=1), "%.4e %.1e %.4e", 3)
            else:
                _array(f, name, v, "%.4e")
        f.write("</PointData>\n")
        f.write("<CellData Scalars='scalars'>\n")
        for name, v in elemental.items():
            if np.issubdtype(np.asarray(v).dtype, np.integer):
                _array(f, name, v, "%d", kind="Int32")
            else:
                _array(f, name, v, "%.4e")
        f.write("</CellData>\n")
        f.write("<Cells>\n")                                                                   # :397-426
        _array(f, "connectivity", icon.T, " ".join(["%d"] * 9), 9, "Int32")
        _array(f, "offsets", (np.arange(nel) + 1) * 9, "%d", kind="Int32")
        _array(f, "types", np.full(nel, 28), "%d", kind="Int32")
        f.write("</Cells>\n")
        f.write("</Piece>\n")
        f.write("</UnstructuredGrid>\n")
        f.write("</VTKFile>\n")


def write_swarm_vtu(path, x, z, fields):
    """output_swarm_to_vtu.py:56-212 for the active particles' arrays given (x, z and every
    field already restricted to the active particles)."""
    n = len(x)
    with open(path, "w") as f:
        f.write("<VTKFile type='UnstructuredGrid' version='0.1' byte_order='BigEndian'> \n")
        f.write("<UnstructuredGrid> \n")
        f.write("<Piece NumberOfPoints=' %5d ' NumberOfCells=' %5d '> \n" % (n, n))
        f.write("<Points> \n")
        f.write("<DataArray type='Float32' NumberOfComponents='3' Format='ascii'> \n")
        np.stack([x, np.zeros(n), z], axis=1).tofile(f, sep=" ")
        f.write("</DataArray>\n")
        f.write("</Points> \n")
        f.write("<PointData Scalars='scalars'>\n")
        for name, v in fields.items():
            if np.issubdtype(np.asarray(v).dtype, np.integer):
                _array(f, name, v, "%d", kind="Int32")
            else:
                _array(f, name, v, "%.3e")
        f.write("</PointData>\n")
        f.write("<Cells>\n")                                                                   # :190-205
        _array(f, "connectivity", np.arange(0, n + 1, dtype=np.int32), "%d", kind="Int32")
        _array(f, "offsets", np.arange(1, n + 2, dtype=np.int32), "%d", kind="Int32")
        _array(f, "types", np.ones(n + 1, dtype=np.int32), "%d", kind="Int32")
        f.write("</Cells>\n")
        f.write("</Piece>\n")
        f.write("</UnstructuredGrid>\n")
        f.write("</VTKFile>\n")


def write_swarm_ascii(path, columns):
    """output_swarm_to_ascii.py:46-104: one row per active particle, the columns given."""
    np.savetxt(path, np.stack(columns, axis=1))


class Pvd:
    """write_in_pvd_files.py:8-39: a ParaView collection, one entry per written file."""

    def __init__(self, path):
        self.f = open(path, "w")
        self.f.write('<?xml version="1.0"?> \n')
        self.f.write('<VTKFile type="Collection" version="0.1" ByteOrder="LittleEndian"> \n')
        self.f.write("  <Collection> \n")
        self.f.flush()

    def add(self, time, file):
        self.f.write('    <DataSet timestep="%s" group="" part="0" file="%s"/>  \n' % (time, file))
        self.f.flush()

    def close(self):
        self.f.write("  </Collection> \n</VTKFile> \n")
        self.f.close()


# ---------------------------------------------------------------------------------------- stream
class OutputStream:
    """Writes a GPUModel's solution (and swarm) every `every_solution` (`every_swarm`) steps into
    `folder`, without stalling the time step: ``submit(istep, time)`` after a step snapshots the
    fields on the model's stream and returns; a side stream and a writer thread do the rest.
    ``close()`` waits for every pending file.  The file names, formats and fields follow the
    reference's writers (solution_%04d.vtu, SWARM/swarm_%04d.vtu[, .ascii], *.pvd)."""

    def __init__(self, model, folder, every_solution=1, every_swarm=1, swarm_ascii=False):
        self.m, self.folder = model, folder
        self.every_solution, self.every_swarm, self.swarm_ascii = every_solution, every_swarm, swarm_ascii
        os.makedirs(os.path.join(folder, "SWARM"), exist_ok=True)
        cfg = model.cfg
        nnx, nnz = 2 * cfg.nelx + 1, 2 * cfg.nelz + 1
        j, i = np.meshgrid(np.arange(nnz), np.arange(nnx), indexing="ij")
        self.x_V = i.ravel() * model.box.hx / 2                  # build_velocity_mesh.py:116-117
        self.z_V = j.ravel() * model.box.hz / 2
        self.side = torch.cuda.Stream()
        self.slots = [self._slot(), self._slot()]
        # a slot is reused once the writer thread is done with its host buffers (waiting only for its
        # copy to the host let a new snapshot overwrite a file's data while the file was written)
        self.free = [threading.Event(), threading.Event()]
        for f in self.free:
            f.set()
        self.next = 0
        self.pvd_sol = Pvd(os.path.join(folder, "solution.pvd"))
        self.pvd_swarm = Pvd(os.path.join(folder, "swarm.pvd"))
        self.q = queue.Queue()
        self.error = None
        self.th = threading.Thread(target=self._writer, daemon=True)
        self.th.start()

    def _sources(self):
        m = self.m
        src = {"u": m.u, "w": m.w, "q": m.q, "T": m.T, "exx": m.exx_n, "ezz": m.ezz_n, "exz": m.exz_n,
               "rho_n": m.nodal["rho"], "eta_n": m.nodal["eta"], "rho_e": m.rho_e, "eta_e": m.eta_e,
               "counts": m.counts, "x": m.x, "z": m.z, "active": m.active, "mat": m.mat,
               "srho": m.props["rho"], "seta": m.props["eta"], "sT": m.props["T"], "up": m.up, "wp": m.wp}
        if m.cfg.solve_T:
            src["qx"], src["qz"] = m.hf[2], m.hf[3]
        return src

    def _slot(self):
        dev = {k: torch.empty_like(v) for k, v in self._sources().items()}
        host = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True) for k, v in dev.items()}
        return dev, host

    def submit(self, istep, time):
        """Queue the output of step `istep` (model time `time`) if the frequencies ask for it."""
        if self.error:
            raise self.error
        sol = istep % self.every_solution == 0
        sw = istep % self.every_swarm == 0
        if not (sol or sw):
            return
        k = self.next
        self.next ^= 1
        self.free[k].wait()                                       # the slot's previous files are written
        self.free[k].clear()
        dev, host = self.slots[k]
        cur = torch.cuda.current_stream()
        for name, v in self._sources().items():                   # device snapshot, on the step's stream
            dev[name].copy_(v, non_blocking=True)
        snap = torch.cuda.Event()
        snap.record(cur)
        with torch.cuda.stream(self.side):
            self.side.wait_event(snap)
            for name in dev:
                host[name].copy_(dev[name], non_blocking=True)
            done = torch.cuda.Event()
            done.record(self.side)
        self.q.put((k, istep, time, sol, sw, host, done))

    def _writer(self):
        while True:
            item = self.q.get()
            if item is None:
                return
            k = item[0]
            try:
                self._write(*item[1:])
            except Exception as ex:                               # reported by the next submit / close
                self.error = ex
            finally:
                self.free[k].set()

    def _write(self, istep, time, sol, sw, host, done):
        done.synchronize()
        h = {k: v.numpy() for k, v in host.items()}
        cfg = self.m.cfg
        if sol:
            nodal = {"Velocity": ("vector", h["u"], h["w"]), "Pressure": h["q"]}
            if cfg.solve_T:
                nodal["Temperature"] = h["T"]
                nodal["Heat flux"] = ("vector", h["qx"], h["qz"])
            nodal.update({"exx": h["exx"], "ezz": h["ezz"], "exz": h["exz"], "Density (nodal)": h["rho_n"],
                          "Viscosity (nodal)": h["eta_n"]})
            elemental = {"Density (elemental)": h["rho_e"], "Viscosity (elemental)": h["eta_e"],
                         "nb particles": h["counts"]}
            name = "solution_%04d.vtu" % istep
            write_solution_vtu(os.path.join(self.folder, name), cfg.nelx, cfg.nelz, self.x_V, self.z_V, nodal,
                               elemental)
            self.pvd_sol.add(time, name)
        if sw:
            a = h["active"].astype(bool)
            fields = {"material": h["mat"][a].astype(np.int32), "Density": h["srho"][a], "Viscosity": h["seta"][a]}
            if cfg.solve_T:
                fields["Temperature"] = h["sT"][a]
            name = "SWARM/swarm_%04d.vtu" % istep
            write_swarm_vtu(os.path.join(self.folder, name), h["x"][a], h["z"][a], fields)
            self.pvd_swarm.add(time, name)
            if self.swarm_ascii:
                write_swarm_ascii(os.path.join(self.folder, "SWARM", "swarm_%04d.ascii" % istep),
                                  [h["x"][a], h["z"][a], h["up"][a], h["wp"][a], h["srho"][a], h["seta"][a]])

    def close(self):
        self.q.put(None)
        self.th.join()
        self.pvd_sol.close()
        self.pvd_swarm.close()
        if self.error:
            raise self.error
