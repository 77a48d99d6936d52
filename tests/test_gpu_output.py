"""Output streamed from device buffers (meeuuw_b200/output.py OutputStream): the files written in
the background while later steps run hold the fields of the step they were submitted at."""
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def arrays(path):
    root = ET.parse(path).getroot()
    return {(a.get("Name") or "points"): np.array(a.text.split(), dtype=float) for a in root.iter("DataArray")}


def test_output_stream_writes_each_submitted_step(tmp_path):
    import torch
    from meeuuw_b200 import configs
    from meeuuw_b200.output import OutputStream
    from meeuuw_b200.timestep import GPUModel
    cfg = configs.blankenbach(16)
    gm = GPUModel(cfg, configs.build_host_model(cfg), stokes="mixed")
    out = OutputStream(gm, str(tmp_path), every_solution=1, every_swarm=2, swarm_ascii=True)
    kept = {}
    for istep in range(3):
        gm.step()
        out.submit(istep, 0.1 * istep)
        kept[istep] = {k: v.detach().cpu().numpy().copy() for k, v in
                       (("u", gm.u), ("T", gm.T), ("q", gm.q), ("x", gm.x), ("act", gm.active), ("eta_e", gm.eta_e))}
    out.close()
    for istep in range(3):
        a = arrays(tmp_path / ("solution_%04d.vtu" % istep))
        k = kept[istep]
        assert np.allclose(a["Velocity"].reshape(-1, 3)[:, 0], k["u"], rtol=1e-4, atol=1e-9 * np.abs(k["u"]).max())
        assert np.allclose(a["Temperature"], k["T"], rtol=1e-4, atol=1e-12)
        assert np.allclose(a["Pressure"], k["q"], rtol=1e-4, atol=1e-9 * np.abs(k["q"]).max())
        assert np.allclose(a["Viscosity (elemental)"], k["eta_e"], rtol=1e-4)
    for istep in (0, 2):
        b = arrays(tmp_path / "SWARM" / ("swarm_%04d.vtu" % istep))
        act = kept[istep]["act"].astype(bool)
        assert np.allclose(b["points"].reshape(-1, 3)[:, 0], kept[istep]["x"][act], rtol=1e-6)
        assert os.path.exists(tmp_path / "SWARM" / ("swarm_%04d.ascii" % istep))
    assert not os.path.exists(tmp_path / "SWARM" / "swarm_0001.vtu")
    files = [d.get("file") for d in ET.parse(tmp_path / "swarm.pvd").getroot().iter("DataSet")]
    assert files == ["SWARM/swarm_0000.vtu", "SWARM/swarm_0002.vtu"]
