"""Drop-in replacements for the reference's per-timestep hot-path functions.

Each module here is named after the reference module whose functions it replaces and exports the
same function names with the same positional signatures and return tuples:

    build_matrix_stokes.build_matrix_stokes
    build_matrix_energy.build_matrix_energy
    locate_particles.locate_particles
    pic_functions.locate_particles___box, interpolate_field_on_particles, advect_particles___box,
                  project_particles_on_elements, project_particle_field_on_nodes_{1,2,3,4},
                  compute_ls_coefficients_P1, compute_ls_coefficients_Q1, population_control
    project_nodal_field_onto_qpoints.project_nodal_{P,V,T}field_onto_qpoints
    uzawa3_solver_L2.uzawa3_solver_L2, cd_u_eta.cd_u_eta
    compute_pressure_offset.compute_pressure_offset
    compute_nodal_pressure.compute_nodal_pressure
    compute_strain_rate.compute_nodal_strain_rate
    compute_nodal_heat_flux.compute_nodal_heat_flux
    postprocessors.compute_global_quantities, compute_Nu

The reference's driver star-imports these modules (``from pic_functions import *`` and so on).
``install()`` puts the device functions into the reference's modules before the driver imports
them, so the driver's own code runs unchanged on top of the device kernels; the reference's
other functions (set-up, output, the annulus geometries) stay as they are.
"""
import importlib

TABLE = {
    "build_matrix_stokes": ["build_matrix_stokes"],
    "build_matrix_energy": ["build_matrix_energy"],
    "locate_particles": ["locate_particles"],
    "pic_functions": ["locate_particles___box", "interpolate_field_on_particles", "advect_particles___box",
                      "project_particles_on_elements", "project_particle_field_on_nodes_1",
                      "project_particle_field_on_nodes_2", "project_particle_field_on_nodes_3",
                      "project_particle_field_on_nodes_4", "compute_ls_coefficients_P1",
                      "compute_ls_coefficients_Q1", "population_control"],
    "project_nodal_field_onto_qpoints": ["project_nodal_Pfield_onto_qpoints", "project_nodal_Vfield_onto_qpoints",
                                         "project_nodal_Tfield_onto_qpoints"],
    "uzawa3_solver_L2": ["uzawa3_solver_L2"],
    "cd_u_eta": ["cd_u_eta"],
    "compute_pressure_offset": ["compute_pressure_offset"],
    "compute_nodal_pressure": ["compute_nodal_pressure"],
    "compute_strain_rate": ["compute_nodal_strain_rate"],
    "compute_nodal_heat_flux": ["compute_nodal_heat_flux"],
    "postprocessors": ["compute_global_quantities", "compute_Nu"],
}


def functions():
    """{(reference module, name): device function} for every entry of TABLE."""
    out = {}
    for mod, names in TABLE.items():
        shim = importlib.import_module(f"{__name__}.{mod}")
        for n in names:
            out[(mod, n)] = getattr(shim, n)
    return out


def install(modules=None):
    """Replace the hot-path functions inside the reference's modules (imported by name from
    sys.path, or taken from `modules`, a {name: module} mapping).  Modules that already imported
    one of these names from another module (``locate_particles`` imports ``pic_functions``) get the
    device function too.  Returns the list of (module, name) pairs replaced."""
    fns = functions()
    done = []
    for (mod, name), fn in fns.items():
        m = (modules or {}).get(mod) or importlib.import_module(mod)
        setattr(m, name, fn)
        done.append((mod, name))
    for mod in TABLE:
        m = (modules or {}).get(mod) or importlib.import_module(mod)
        for (_, name), fn in fns.items():
            if hasattr(m, name):
                setattr(m, name, fn)
    return done
