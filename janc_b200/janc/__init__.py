"""Drop-in mirror of JANC's ``janc_v2`` modules for the per-step path.

Replace ``janc_v2`` by ``janc_b200.janc`` in imports: the same module paths,
function names, arguments and configuration dictionaries, with the compute in
``libjanc_b200.so``.  Like the reference, configuration lives in module state
set by ``set_thermo``/``set_reaction``/``set_flux_solver``/``set_boundary`` (or
``Simulator``); arrays may be torch CUDA tensors (returned as such) or NumPy
arrays (returned as NumPy).  ``simulation_config['precision']`` (an extension)
selects ``fp64`` (default), ``fp64_strict`` or ``mixed``.
"""
