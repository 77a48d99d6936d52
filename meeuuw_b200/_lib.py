"""ctypes binding of ``libmeeuuw_b200.so`` (the C ABI declared in ``include/meeuuw_b200.h``).

There is no fallback: if the shared library is missing or no CUDA device is present, every
entry point raises.  Device memory is owned by torch tensors; only raw pointers cross the ABI.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmeeuuw_b200.so")

MW_OK = 0
STATUS = {0: "MW_OK", 1: "MW_ERR_BAD_ARG", 2: "MW_ERR_CUDA", 3: "MW_ERR_NOT_CONVERGED", 4: "MW_ERR_WORKSPACE",
          5: "MW_ERR_DEVICE_FLAG"}
FLAG_R_OUT, FLAG_T_OUT, FLAG_ELEMENT_RANGE, FLAG_EMPTY_ELEMENT, FLAG_NONFINITE, FLAG_ITER_LIMIT = 1, 2, 4, 8, 16, 32
FLAG_POP_UNAVAILABLE, FLAG_POP_MASK_EMPTY, FLAG_POP_DRAWS = 64, 128, 256
MAX_FIELDS = 8
AVG = {"arithmetic": 0, "geometric": 1, "harmonic": 2}
SPACE_Q2, SPACE_Q1_ON_V, SPACE_Q1 = 0, 1, 2
MATERIAL_BOUSSINESQ, MATERIAL_TWO = 0, 1

c_void_p, c_int32, c_int64, c_double, c_size_t = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_size_t
c_uint64 = ctypes.c_uint64


class MwBox(ctypes.Structure):
    _fields_ = [("nelx", c_int32), ("nelz", c_int32), ("Lx", c_double), ("Lz", c_double), ("hx", c_double),
                ("hz", c_double)]


class MwMaterial(ctypes.Structure):
    _fields_ = [("kind", c_int32), ("rho0", c_double), ("alphaT", c_double), ("fk_gamma", c_double),
                ("eta0", c_double), ("hcond", c_double), ("hcapa", c_double), ("hprod", c_double),
                ("mat_rho", c_double * 8), ("mat_eta", c_double * 8)]


class MwStokesIn(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("rhoq", "etaq", "JxWq", "jcbi00q", "jcbi01q", "jcbi10q", "jcbi11q", "gxq",
                                        "gzq", "eta_e", "N_V", "N_P", "dNdr_V", "dNdt_V", "dNdr_P", "dNdt_P",
                                        "bc_fix_V", "bc_val_V")] + [("eta_ref", c_double), ("L_ref", c_double)]


class MwStokesOut(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("VV_Stokes", "VV_K", "VV_G", "VV_GT", "VV_M", "VV_M_eta", "VV_H", "rhs_f",
                                        "rhs_h")]


class MwEnergyIn(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("T", "rhoq", "etaq", "Tq", "uq", "wq", "hcondq", "hcapaq", "alphaq",
                                        "hprodq", "exxq", "ezzq", "exzq", "JxWq", "jcbi00q", "jcbi01q", "jcbi10q",
                                        "jcbi11q", "N_T", "dNdr_T", "dNds_T", "bc_fix_T", "bc_val_T")] + \
        [("dt", c_double), ("rho0", c_double), ("dt_dev", c_void_p), ("formulation", c_int32)]


class MwGauss3(ctypes.Structure):
    _fields_ = [("c", c_double * 3), ("w", c_double * 3)]


class MwDtParams(ctypes.Structure):
    _fields_ = [("CFLnb", c_double), ("hx", c_double), ("hz", c_double), ("dt_max", c_double), ("solve_T", c_int32)]


class MwNodal5(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("exx", "ezz", "exz", "q", "T")]


class MwSwarmProps(ctypes.Structure):
    _fields_ = [(k, c_void_p) for k in ("exx", "ezz", "exz", "p", "T", "rho", "eta", "hcond", "hcapa", "hprod",
                                        "alpha")]


_lib = None

class MwLsFields(ctypes.Structure):
    _fields_ = [("phi", c_void_p * 8), ("coef", c_void_p * 8), ("fmin", c_void_p * 8), ("fmax", c_void_p * 8),
                ("n", c_int32)]


class MwPcFields(ctypes.Structure):
    _fields_ = [("f", c_void_p * 8), ("n", c_int32)]


# name -> (restype, argtypes)
_PROTOS = {
    "mw_locate_box": (c_int32, [MwBox, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_void_p]),
    "mw_interp_q2": (c_int32, [MwBox, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                               c_void_p, c_void_p]),
    "mw_interp_material": (c_int32, [MwBox, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, MwNodal5,
                                     MwMaterial, MwSwarmProps, c_void_p]),
    "mw_advect_box": (c_int32, [MwBox, c_int32, c_double, c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_bin_workspace_bytes": (c_size_t, [c_int32]),
    "mw_bin_particles": (c_int32, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_size_t, c_void_p, c_void_p]),
    "mw_project_elements": (c_int32, [c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                                      c_void_p, c_void_p, c_void_p]),
    "mw_project_nodes_workspace_bytes": (c_size_t, [MwBox, c_int32]),
    "mw_project_nodes": (c_int32, [MwBox, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "mw_nodal_to_qpoints": (c_int32, [MwBox, c_int32, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_ls_fit": (c_int32, [MwBox, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, MwLsFields, c_double, c_void_p,
                            c_void_p]),
    "mw_ls_to_qpoints": (c_int32, [MwBox, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_population_workspace_bytes": (c_size_t, [c_int32, c_int64]),
    "mw_population_control": (c_int32, [MwBox, c_int32, c_int64] + [c_void_p] * 11 + [MwPcFields, c_void_p, c_int64,
                                        c_uint64, c_void_p, c_void_p, c_size_t, c_void_p, c_void_p]),
    "mw_assemble_stokes_workspace_bytes": (c_size_t, [MwBox]),
    "mw_assemble_stokes": (c_int32, [MwBox, c_int32, c_int32, MwStokesIn, MwStokesOut, c_void_p, c_size_t, c_void_p]),
    "mw_stokes_rhs_body": (c_int32, [MwBox, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_size_t, c_void_p]),
    "mw_assemble_energy_workspace_bytes": (c_size_t, [MwBox]),
    "mw_assemble_energy": (c_int32, [MwBox, c_int32, MwEnergyIn, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "mw_post_workspace_bytes": (c_size_t, []),
    "mw_pressure_offset": (c_int32, [MwBox, c_int32, c_void_p, c_void_p, c_void_p, c_double, c_void_p, c_void_p,
                                     c_size_t, c_void_p]),
    "mw_nodal_pressure": (c_int32, [MwBox, c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p]),
    "mw_nodal_strain_rate": (c_int32, [MwBox] + [c_void_p] * 12),
    "mw_nodal_heat_flux": (c_int32, [MwBox] + [c_void_p] * 12),
    "mw_nu_workspace_bytes": (c_size_t, [MwBox]),
    "mw_compute_nu": (c_int32, [MwBox, c_void_p, c_void_p, c_void_p, c_void_p, MwGauss3, c_void_p, c_void_p,
                                c_size_t, c_void_p]),
    "mw_global_quantities": (c_int32, [c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                                       c_void_p, c_void_p, c_size_t, c_void_p]),
    "mw_compute_dt": (c_int32, [c_int64, c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, MwDtParams,
                                c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "mw_split_solution": (c_int32, [c_int64, c_int64, c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p,
                                    c_void_p]),
    "mw_elemental_to_qpoints": (c_int32, [c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_energy_matvec": (c_int32, [MwBox, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_energy_solve_workspace_bytes": (c_size_t, [MwBox]),
    "mw_energy_device_info": (c_int32, [MwBox, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_energy_solve": (c_int32, [MwBox, c_void_p, c_void_p, c_void_p, c_double, c_int32, c_void_p, c_void_p,
                                  c_void_p, c_size_t, c_void_p]),
    "mw_coo_length": (c_int64, [MwBox, c_int32]),
    "mw_coo_pattern": (c_int32, [MwBox, c_int32, c_void_p, c_void_p, c_void_p]),
    "mw_csr_rows": (c_int64, [MwBox, c_int32]),
    "mw_csr_workspace_bytes": (c_size_t, [MwBox, c_int32]),
    "mw_csr_pattern": (c_int32, [MwBox, c_int32, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "mw_csr_columns": (c_int32, [MwBox, c_int32, c_void_p, c_void_p, c_void_p]),
    "mw_csr_values": (c_int32, [MwBox, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_energy_op_bytes": (c_size_t, [MwBox]),
    "mw_energy_op_setup": (c_int32, [MwBox, MwEnergyIn, c_void_p, c_size_t, c_void_p, c_void_p]),
    "mw_energy_op_apply": (c_int32, [MwBox, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mw_energy_op_solve_workspace_bytes": (c_size_t, [MwBox]),
    "mw_energy_op_solve": (c_int32, [MwBox, c_void_p, c_void_p, c_void_p, c_double, c_int32, c_void_p, c_void_p,
                                     c_void_p, c_size_t, c_void_p]),
}


def extra_protos(d):
    """Other modules register their prototypes here (applied now if the library is loaded)."""
    _PROTOS.update(d)
    if _lib is not None:
        for name, (res, args) in d.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args


def lib():
    """Load the shared library (once).  Raises if it is missing: there is no CPU path."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m meeuuw_b200.build` "
                               "(the CUDA library is required; there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return sorted(_PROTOS)


def ptr(t):
    """Raw device pointer of a CUDA tensor (or None)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("meeuuw_b200 kernels take CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def call(name, *args):
    """Call an entry point and raise on a non-zero status."""
    fn = getattr(lib(), name)
    rc = fn(*args)
    if isinstance(rc, int) and fn.restype is c_int32 and rc != MW_OK:
        raise RuntimeError(f"{name} returned {STATUS.get(rc, rc)}")
    return rc


def ptr_array(tensors):
    """HOST array of device pointers (for the multi-field entry points)."""
    arr = (c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])
    return arr


def box_of(nelx, nelz, Lx, Lz):
    return MwBox(int(nelx), int(nelz), float(Lx), float(Lz), float(Lx) / int(nelx), float(Lz) / int(nelz))


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("meeuuw_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
