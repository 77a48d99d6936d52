"""Host-side checks of the drop-in layer (no GPU): the functions have the reference's positional
signatures (recorded from the reference in tests/golden/signatures.json), install() swaps them
into the reference's modules, and only the uniform box numbering is accepted."""
import inspect
import json
import os
import types

import numpy as np
import pytest

from oracle.fe import BoxMesh

HERE = os.path.dirname(__file__)


def test_signatures_match_reference():
    from meeuuw_b200 import dropin
    with open(os.path.join(HERE, "golden", "signatures.json")) as f:
        ref = json.load(f)
    fns = dropin.functions()
    assert set(f"{m}.{n}" for m, n in fns) == set(ref)
    for (mod, name), fn in fns.items():
        params = inspect.signature(fn).parameters
        positional = [p for p, v in params.items() if v.default is inspect.Parameter.empty]
        assert positional == ref[f"{mod}.{name}"], (mod, name)
        extra = [p for p, v in params.items() if v.default is not inspect.Parameter.empty]
        assert extra in ([], ["V0", "P0"]), (mod, name, extra)


def test_install_replaces_names_in_reference_modules():
    from meeuuw_b200 import dropin
    fakes = {}
    for mod, names in dropin.TABLE.items():
        m = types.ModuleType(mod)
        for n in names:
            setattr(m, n, lambda *a: "reference")
        m.unrelated = "kept"
        fakes[mod] = m
    # a module that imported a pic function by name gets the device function as well
    fakes["locate_particles"].locate_particles___box = lambda *a: "reference"
    done = dropin.install(modules=fakes)
    assert len(done) == sum(len(v) for v in dropin.TABLE.values())
    fns = dropin.functions()
    for (mod, name), fn in fns.items():
        assert getattr(fakes[mod], name) is fn
        assert fakes[mod].unrelated == "kept"
    assert fakes["locate_particles"].locate_particles___box is fns[("pic_functions", "locate_particles___box")]


def test_box_numbering_is_recognised_and_others_refused():
    from meeuuw_b200.dropin import _common as C
    m = BoxMesh(6, 4, 1.5, 1.0)
    assert C.box_dims(m.icon_V, m.nel) == (6, 4)
    C.check_icon_P(m.icon_P, 6, 4)
    C.check_coords(m.x_V, m.z_V, 6, 4, m.hx, m.hz)
    bad = m.icon_V.copy()
    bad[:, [3, 4]] = bad[:, [4, 3]]             # two elements swapped
    with pytest.raises(NotImplementedError):
        C.box_dims(bad, m.nel)
    with pytest.raises(NotImplementedError):
        C.check_coords(m.x_V * 1.01, m.z_V, 6, 4, m.hx, m.hz)
    with pytest.raises(NotImplementedError):
        C.require_box("quarter", False)
    b = C.box(6, 4, m.hx, m.hz)
    assert (b.nelx, b.nelz, b.hx, b.hz) == (6, 4, m.hx, m.hz)


def test_host_mode_and_conversions_without_gpu():
    import torch
    from meeuuw_b200.dropin import _common as C
    assert C.host_mode(np.zeros(3), torch.zeros(2))
    a = np.arange(4.0)
    C.copy_into(a, torch.tensor([4.0, 3.0, 2.0, 1.0], dtype=torch.float64))
    assert np.array_equal(a, [4, 3, 2, 1])
    flags = np.zeros(3, dtype=bool)
    C.copy_into(flags, torch.tensor([1, 0, 1], dtype=torch.uint8))
    assert flags.tolist() == [True, False, True]
