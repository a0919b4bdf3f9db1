"""3-D operators of the B200 particle pass (``tensorsph.threed``)."""
from .kernel3 import (calibrated_particle_mass, cubic_spline_gradient, cubic_spline_kernel,
                      cubic_spline_laplacian, lattice_bias, lattice_kernel_sum, pair_kernels,
                      sigma3)
from .csf3 import CSFState3, csf_fields3, surface_tension_acceleration3
from .neighbors3 import box_pairs, minimum_image, periodic_pairs
from .operators3 import accelerations, tait_density, tait_pressure
from .solver import acoustic_dt, cubic_lattice, hydrostatic_density, wall_shell
from .hydrostatic import HydrostaticResult, build_pressure_profile, run_hydrostatic

__all__ = [
    "CSFState3", "csf_fields3", "surface_tension_acceleration3",
    "accelerations", "box_pairs", "calibrated_particle_mass", "cubic_lattice",
    "cubic_spline_gradient", "cubic_spline_kernel", "cubic_spline_laplacian",
    "hydrostatic_density", "lattice_bias", "lattice_kernel_sum", "minimum_image",
    "pair_kernels", "periodic_pairs", "sigma3", "tait_density", "tait_pressure", "wall_shell",
    "acoustic_dt", "HydrostaticResult", "build_pressure_profile", "run_hydrostatic",
]
