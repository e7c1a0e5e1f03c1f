"""ctypes binding of the C ABI in ``include/janc_b200.h``.

The shared library is built in-tree (``janc_b200/libjanc_b200.so``) by
``janc_b200._build``.  There is no CPU fallback: every compute entry point
needs the library and a CUDA device, and a missing library raises.
"""
import ctypes
import os

from . import mechanism as _mech

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libjanc_b200.so")

BC_KIND = {"periodic": 0, "slip_wall": 1, "zero_gradient": 2, "no_slip_wall": 3,
           "pressure_outlet": 4, "rdc_injector": 5}
BC_HALO = 6  # x side bordering another slab (jb_set_exchange)
XCH_DT, XCH_HALO = 1, 2  # jb_exchange_flags
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p)
PRECISION = {"fp64_strict": 0, "fp64": 1, "mixed": 2}
FLUX_SCHEME = {"LF": 0, "HLLC": 1, "AUSMPW_plus": 2, "SW": 3}  # split method / Riemann solver
RECONSTRUCTION = {"WENO5_JS": 0, "MUSCL": 1}
STATUS = {1: "bad argument", 2: "CUDA error", 4: "non-finite state", 8: "singular chemistry matrix",
          16: "device wait timed out", 32: "unsupported configuration"}

EXPORTS = ["jb_version", "jb_create", "jb_destroy", "jb_set_theta", "jb_flux_func", "jb_update_aux",
           "jb_reaction_source_terms", "jb_advance", "jb_cfl_dt", "jb_get_thermo", "jb_status",
           "jb_workspace_bytes", "jb_set_spacing", "jb_set_flux_scheme", "jb_set_reconstruction", "jb_set_transport", "jb_set_exchange", "jb_set_ghost_cells", "jb_boundary_conditions",
           "jb_sizeof_mech_params",
           "jb_sizeof_grid",
           "jb_last_error", "jb_probe_fp64_fma", "jb_set_kernel_timing", "jb_kernel_times",
           "jb_update_aux_noalloc", "jb_rk3", "jb_u_to_prim",
           "jb_ens_create", "jb_ens_destroy", "jb_ens_instance", "jb_ens_total_cells", "jb_ens_configure",
           "jb_ens_set_back_pressure",
           "jb_ens_autotune", "jb_ens_launch_shape", "jb_ens_advance", "jb_ens_advance_direct",
           "jb_ens_status", "jb_ens_last_error", "jb_ens_selftest_timeout",
           "jb_set_probe", "jb_set_log_A_offset", "jb_record_doubles", "jb_advance_ex", "jb_adjoint_reserve", "jb_adjoint_step",
           "jb_state_from_PTY_vjp", "jb_amr_stage", "jb_amr_chem", "jb_amr_flux",
           "jb_amr_update_aux"]

_lib = None


class JancError(RuntimeError):
    pass


def status_text(code):
    return ", ".join(v for k, v in STATUS.items() if code & k) or "ok"


class Transport(ctypes.Structure):
    """jb_transport (laminar transport model of the viscous fluxes)."""
    _fields_ = [("viscosity_model", ctypes.c_int), ("conductivity_model", ctypes.c_int),
                ("diffusivity_model", ctypes.c_int), ("turbulence_model", ctypes.c_int)] + \
        [(n, ctypes.c_double) for n in ("mu_ref", "T_ref", "S", "nu0", "Pr", "Le", "k0", "D0", "Pr_t", "Le_t")]


def lib(path=None):
    """Load (once) and return the shared library with argument types set."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise JancError(f"janc_b200 native library not found at {p}; build it with "
                        "`python -m janc_b200._build` (nvcc, sm_100a)")
    L = ctypes.CDLL(p)
    vp, dp, i, d, ll = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
    L.jb_version.restype = ctypes.c_char_p
    L.jb_create.argtypes = [ctypes.POINTER(_mech.MechParams), i, i, i, d, d, ctypes.POINTER(ctypes.c_int),
                            i, ctypes.POINTER(vp)]
    L.jb_destroy.argtypes = [vp]
    L.jb_set_theta.argtypes = [vp, d, dp, d]
    L.jb_flux_func.argtypes = [vp, dp, dp, d, dp, vp]
    L.jb_update_aux.argtypes = [vp, dp, dp, dp, vp]
    L.jb_reaction_source_terms.argtypes = [vp, dp, dp, d, dp, vp]
    L.jb_advance.argtypes = [vp, dp, dp, dp, dp, d, d, i, dp, vp]
    L.jb_cfl_dt.argtypes = [vp, dp, dp, d, dp, vp]
    L.jb_rk3.argtypes = [vp, dp, dp, dp, dp, d, vp]
    L.jb_u_to_prim.argtypes = [vp, dp, dp, dp, dp, dp, dp, dp, dp, vp]
    L.jb_get_thermo.argtypes = [vp, ll, dp, dp, dp, dp, dp, dp, dp, vp]
    L.jb_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint), vp]
    L.jb_workspace_bytes.argtypes = [vp]
    L.jb_workspace_bytes.restype = ll
    L.jb_set_spacing.argtypes = [vp, d, d]
    L.jb_set_flux_scheme.argtypes = [vp, i]
    L.jb_set_reconstruction.argtypes = [vp, i]
    L.jb_set_transport.argtypes = [vp, ctypes.POINTER(Transport)]
    L.jb_set_exchange.argtypes = [vp, dp, dp, dp, EXCHANGE_FN, vp]
    L.jb_set_ghost_cells.argtypes = [vp, dp, dp, dp, dp, EXCHANGE_FN, vp]
    L.jb_boundary_conditions.argtypes = [vp, dp, dp, dp, dp, vp]
    L.jb_probe_fp64_fma.argtypes = [i, i, dp, vp]
    L.jb_set_kernel_timing.argtypes = [vp, i]
    L.jb_update_aux_noalloc.argtypes = [ctypes.POINTER(_mech.MechParams), i, i, i, i, dp, dp, dp, vp]
    L.jb_kernel_times.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
    L.jb_last_error.argtypes = [vp]
    L.jb_last_error.restype = ctypes.c_char_p
    ip, dpp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    L.jb_ens_create.argtypes = [ctypes.POINTER(_mech.MechParams), i, ip, dpp, ip, dpp, dpp, i, ctypes.POINTER(vp)]
    L.jb_ens_destroy.argtypes = [vp]
    L.jb_ens_instance.argtypes = [vp, i, ctypes.POINTER(vp), ctypes.POINTER(vp), ip]
    L.jb_ens_total_cells.argtypes = [vp]
    L.jb_ens_total_cells.restype = ll
    L.jb_ens_configure.argtypes = [vp, i, i]
    L.jb_ens_set_back_pressure.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.jb_ens_autotune.argtypes = [vp, i, vp, ip, ip, dpp]
    L.jb_ens_launch_shape.argtypes = [vp, ip, ip, ip, ip, ip]
    L.jb_ens_advance.argtypes = [vp, i, dp, vp]
    L.jb_ens_advance_direct.argtypes = [vp, i, dp, vp]
    L.jb_ens_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(ctypes.c_uint), vp]
    L.jb_set_probe.argtypes = [vp, i, i, i, i]
    L.jb_set_log_A_offset.argtypes = [vp, dpp]
    L.jb_record_doubles.argtypes = [vp]
    L.jb_record_doubles.restype = ll
    L.jb_advance_ex.argtypes = [vp, dp, dp, dp, dp, d, d, i, dp, dp, dp, dp, vp]
    L.jb_adjoint_reserve.argtypes = [vp]
    L.jb_adjoint_step.argtypes = [vp, dp, dp, d, dp, dp, dp, dp, dp, vp]
    L.jb_state_from_PTY_vjp.argtypes = [vp, dp, dp, dp, dp, dp, dp, vp]
    L.jb_amr_stage.argtypes = [vp, i, i, i, d, d, i, dp, dp, d, dp, vp]
    L.jb_amr_chem.argtypes = [vp, i, i, i, dp, d, dp, vp]
    L.jb_amr_flux.argtypes = [vp, i, i, i, d, d, dp, dp, d, dp, vp]
    L.jb_amr_update_aux.argtypes = [vp, i, i, i, dp, dp, dp, vp]
    L.jb_ens_selftest_timeout.argtypes = [vp, d, ctypes.POINTER(ctypes.c_uint), vp]
    L.jb_ens_last_error.argtypes = [vp]
    L.jb_ens_last_error.restype = ctypes.c_char_p
    for name in EXPORTS:
        getattr(L, name)
    if L.jb_sizeof_mech_params() != ctypes.sizeof(_mech.MechParams):
        raise JancError("jb_mech_params layout mismatch between Python and the library")
    _lib = L
    return L


def check(rc, handle=None, what="", ensemble=False):
    if rc != 0:
        msg = ""
        if handle is not None:
            err = lib().jb_ens_last_error if ensemble else lib().jb_last_error
            msg = err(handle).decode()
        raise JancError(f"{what} failed: {status_text(rc)} (code {rc}) {msg}".strip())
