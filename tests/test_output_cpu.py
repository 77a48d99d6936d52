"""The VTU / ASCII / PVD writers (meeuuw_b200/output.py) on host arrays: well-formed XML, the
reference's array names and cell layout (output_solution_to_vtu.py, output_swarm_to_vtu.py,
write_in_pvd_files.py), values read back within the ASCII formats' precision."""
import os
import xml.etree.ElementTree as ET

import numpy as np

from meeuuw_b200 import output


def arrays(path):
    root = ET.parse(path).getroot()
    return {(a.get("Name") or "points"): np.array(a.text.split(), dtype=float) for a in root.iter("DataArray")}


def test_q2_connectivity_matches_the_host_model():
    from meeuuw_b200 import configs
    host = configs.build_host_model(configs.blankenbach(5, nelz=3))
    assert np.array_equal(output.q2_connectivity(5, 3), host.icon_V)


def test_solution_and_swarm_files_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    nelx, nelz = 4, 3
    nn = (2 * nelx + 1) * (2 * nelz + 1)
    x = np.tile(np.arange(2 * nelx + 1) * 0.125, 2 * nelz + 1)
    z = np.repeat(np.arange(2 * nelz + 1) * 0.1, 2 * nelx + 1)
    u, w, q = rng.standard_normal(nn), rng.standard_normal(nn), rng.standard_normal(nn)
    p = tmp_path / "solution_0000.vtu"
    output.write_solution_vtu(str(p), nelx, nelz, x, z, {"Velocity": ("vector", u, w), "Pressure": q},
                              {"nb particles": np.arange(nelx * nelz, dtype=np.int32)})
    a = arrays(p)
    pts = a["points"].reshape(-1, 3)
    assert np.allclose(pts[:, 0], x, rtol=1e-5) and np.allclose(pts[:, 2], z, rtol=1e-5)
    vel = a["Velocity"].reshape(-1, 3)
    assert np.allclose(vel[:, 0], u, rtol=1e-4, atol=1e-12) and np.allclose(vel[:, 2], w, rtol=1e-4, atol=1e-12)
    assert np.allclose(a["Pressure"], q, rtol=1e-4, atol=1e-12)
    assert np.array_equal(a["connectivity"].reshape(-1, 9), output.q2_connectivity(nelx, nelz).T)
    assert np.all(a["types"] == 28) and np.array_equal(a["offsets"], 9 * (np.arange(nelx * nelz) + 1))
    n = 50
    sx, sz, rho = rng.uniform(size=n), rng.uniform(size=n), rng.uniform(1, 2, n)
    ps = tmp_path / "swarm_0000.vtu"
    output.write_swarm_vtu(str(ps), sx, sz, {"Density": rho, "material": np.ones(n, dtype=np.int32)})
    b = arrays(ps)
    assert np.allclose(b["points"].reshape(-1, 3)[:, 0], sx) and np.allclose(b["Density"], rho, rtol=1e-3)
    assert np.all(b["types"] == 1) and len(b["connectivity"]) == n + 1
    pv = output.Pvd(str(tmp_path / "solution.pvd"))
    pv.add(0.5, "solution_0000.vtu")
    pv.close()
    root = ET.parse(tmp_path / "solution.pvd").getroot()
    assert [d.get("file") for d in root.iter("DataSet")] == ["solution_0000.vtu"]
