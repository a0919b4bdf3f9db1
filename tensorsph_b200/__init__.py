"""B200-native particle pass of TensorSPH: linked-cell pair search with its
Verlet skin cache and the WCSPH pair pass, as hand-written sm_100a CUDA behind
the reference's Python API (``tensorsph.neighbor_search``,
``tensorsph.droplet_impact.rhs``, ``tensorsph.dam_break_3d.rhs_3d``,
``tensorsph.threed.accelerations``, ``tensorsph.particle_shifting``)."""

__version__ = "0.1.0"
