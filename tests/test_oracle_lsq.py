"""The least-squares / limiter / population-control oracle against the reference's own outputs
(``tests/golden/lsq.npz``, ``population.npz``, made by ``make_golden.py lsq``).

Normal equations are summed in the reference's order and solved with the same LAPACK solve, so
coefficients agree to round-off (1e-12 relative); element extrema, the limiter's output, element
indices, active flags and material ids are exact.
"""
import numpy as np
import pytest

from conftest import golden, rel_err


@pytest.fixture(scope="module")
def M():
    return golden("mesh_6x4")


@pytest.mark.parametrize("order", [3, 4])
def test_ls_coefficients(M, order):
    from oracle import lsq
    g = golden("lsq")
    nel = 24
    coefs, fmin, fmax = lsq.ls_coefficients(order, nel, g["x_e"], g["z_e"], g["swarm_x"], g["swarm_z"],
                                            g["swarm_iel"], [g["swarm_rho"], g["swarm_eta"]])
    tag = "P1" if order == 3 else "Q1"
    for f, name in enumerate(("rho", "eta")):
        for j, c in enumerate("abcd"[:order]):
            assert rel_err(coefs[f][:, j], g[f"out_{tag}_{name}_{c}"]) < 1e-12, (name, c)
        assert np.array_equal(fmin[f], g[f"out_{tag}_{name}_min"])
        assert np.array_equal(fmax[f], g[f"out_{tag}_{name}_max"])
        if order == 3:
            lim = lsq.limit_p1(coefs[f], fmin[f], fmax[f], float(M["hx"]))
            assert rel_err(lim[:, 1], g[f"out_P1lim_{name}_b"]) < 1e-12
            assert rel_err(lim[:, 2], g[f"out_P1lim_{name}_c"]) < 1e-12
            q = lsq.ls_to_qpoints(lim, M["xq"], M["zq"], g["x_e"], g["z_e"])
            assert rel_err(q, g[f"out_P1_{name}q"]) < 1e-12
        else:
            q = lsq.ls_to_qpoints(coefs[f], M["xq"], M["zq"], g["x_e"], g["z_e"])
            assert rel_err(q, g[f"out_Q1_{name}q"]) < 1e-12


def test_limiter():
    from oracle import lsq
    g = golden("lsq")
    out = np.array([lsq.limiter(g["lim_c0"][i], g["lim_c1"][i], g["lim_c2"][i], g["lim_S"][i], g["lim_L"][i],
                                float(g["lim_h"])) for i in range(len(g["lim_c0"]))])
    assert np.array_equal(out, g["out_lim"])


def _arrays(g):
    return {k: g[k].copy() for k in ("swarm_active", "swarm_iel", "swarm_r", "swarm_t", "swarm_x", "swarm_z",
                                     "swarm_u", "swarm_w", "swarm_eta", "swarm_mat")}


def test_population_control(M):
    from oracle import lsq
    g = golden("population")
    a = _arrays(g)
    n = lsq.population_control(M["x_V"], M["z_V"], M["icon_V"], 24, int(g["nparticle_min"]), g["nparticle_e"],
                               a["swarm_active"], a["swarm_iel"], a["swarm_r"], a["swarm_t"], a["swarm_x"],
                               a["swarm_z"], a["swarm_u"], a["swarm_w"], a["swarm_eta"], a["swarm_mat"], g["draws"])
    assert n == int(g["needed"]) > 0
    for k in ("swarm_active", "swarm_iel", "swarm_mat", "swarm_r", "swarm_t"):
        assert np.array_equal(a[k], g["out_" + k]), k
    for k in ("swarm_x", "swarm_z", "swarm_u", "swarm_w", "swarm_eta"):
        assert rel_err(a[k], g["out_" + k]) < 1e-14, k


def test_population_control_errors(M):
    from oracle import lsq
    g = golden("population")
    a = _arrays(g)
    args = lambda ne, act: (M["x_V"], M["z_V"], M["icon_V"], 24, 7, ne, act, a["swarm_iel"], a["swarm_r"],
                            a["swarm_t"], a["swarm_x"], a["swarm_z"], a["swarm_u"], a["swarm_w"], a["swarm_eta"],
                            a["swarm_mat"], g["draws"])
    with pytest.raises(ValueError, match="not available yet"):
        lsq.population_control(*args(np.zeros(24, dtype=np.int32), a["swarm_active"].copy()))
    act = a["swarm_active"].copy()
    act[a["swarm_iel"] == 3] = False                                   # a flagged element left empty
    with pytest.raises(ValueError, match="mask empty"):
        lsq.population_control(*args(g["nparticle_e"], act))
