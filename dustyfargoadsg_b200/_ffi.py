"""ctypes view of the C ABI declared in include/fargo_b200.h.

The structures mirror the C layout field for field; `check_layout()` compares
their sizes with the library's own `fb_struct_size`.  Loading fails loudly
when libfargo_b200.so has not been built: there is no CPU fallback.
"""
import ctypes as C
import os

FB_MAX_PLANETS = 16
FB_OK = 0
FB_ERR_NEGATIVE = -6  # the crash test fired during a DT that still completed
FB_ERR = {
    -1: "FB_ERR_INVALID", -2: "FB_ERR_UNSUPPORTED", -3: "FB_ERR_CUDA", -4: "FB_ERR_NOMEM",
    -5: "FB_ERR_NAN", -6: "FB_ERR_NEGATIVE", -7: "FB_ERR_SUBSTEPS", -8: "FB_ERR_TIMEOUT",
    -9: "FB_ERR_IO", -10: "FB_ERR_STATE", -11: "FB_ERR_NODEVICE",
}
FB_F_DENS, FB_F_VRAD, FB_F_VTHETA, FB_F_ENERGY, FB_F_ALL = 1, 2, 4, 8, 15
FB_STAGE_TRANSPORT, FB_STAGE_VISCOSITY, FB_STAGE_BOUNDARY, FB_STAGE_DAMPING, FB_STAGE_SELFGRAV = 1, 2, 3, 4, 5

_D = C.c_double
_I = C.c_int
_P = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)
_NP = FB_MAX_PLANETS


class FbParams(C.Structure):
    _fields_ = [
        ("nrad", _I), ("nsec", _I), ("rmin", _D), ("rmax", _D), ("log_grid", _I),
        ("pmin", _D), ("pmax", _D),
        ("dt", _D), ("ntot", _I), ("ninterm", _I),
        ("sigma0", _D), ("sigmaslope", _D), ("aspectratio", _D), ("flaringindex", _D),
        ("alphaviscosity", _D), ("viscosity", _D),
        ("adiabaticindex", _D), ("energy_equation", _I), ("viscous_heating", _I),
        ("beta_cooling", _I), ("betacoolingtime", _D), ("betacoolingslope", _D),
        ("thermal_cooling", _I), ("constant_opacity", _I), ("imposedconstantopacity", _D),
        ("factoropacities", _D), ("stellar_irradiation", _I), ("backgroundtemperature", _D),
        ("slopebackgroundtemperature", _D), ("stellarluminosity", _D),
        ("self_gravity", _I), ("sgthicknesssmoothing", _D),
        ("thicknesssmoothing", _D), ("rochesmoothing", _D), ("indirecttermsmoothing", _D),
        ("masstaper", _D), ("omegaframe", _D),
        ("indirect_term", _I), ("discard_gas_indirect_term", _I), ("alternative_gas_indirect_term", _I),
        ("forced_circular", _I), ("exclude_hill", _I),
        ("excludehillfactor", _D), ("eccentricity", _D), ("releasedate", _D), ("releaseradius", _D),
        ("fast_transport", _I), ("wall_boundary", _I), ("evanescent", _I),
        ("wkzrmin", _D), ("wkzrmax", _D), ("dampingtodynamicaltimeratio", _D),
        ("damp_to_axi", _I), ("damp_to_ini", _I), ("add_floors", _I),
        ("densityfloor", _D), ("zero_vrad_bc", _I), ("open_inner", _I), ("kn_open", _I),
        ("non_reflecting", _I),
        ("mindt", _D), ("maxdt", _D), ("imposeddiskdrift", _D),
        ("factorunitmass", _D), ("factorunitlength", _D), ("factormmw", _D),
        ("nbpart", _I),
        ("sizeminpart", _D), ("sizemaxpart", _D), ("sizepartslope", _D), ("rhopart", _D), ("dustslope", _D),
        ("rmindust", _D), ("rmaxdust", _D),
        ("dust_feel_disk", _I), ("dust_feel_planets", _I), ("dust_feel_turb", _I), ("dust_feedback", _I),
        ("dust_feel_sg", _I),
        ("sfta", _I), ("interpolation", _I), ("write_dust_density", _I),
        ("unsupported", C.c_ulonglong),
        ("planetconfig", C.c_char * 512), ("outputdir", C.c_char * 512),
        ("mhd_lsa", _I), ("nbturbmodes", _I), ("high_m_cutoff", _I),
        ("gammaturb", _D), ("lsamodespeedup", _D), ("turbrmin", _D), ("turbrmax", _D),
        ("cavityradius", _D), ("cavityratio", _D), ("cavitywidth", _D),
        ("entropy_diffusion", _I), ("radiative_diffusion", _I), ("diffusivity", _D),
        ("corotating", _I), ("add_noise", _I), ("temppresc", _I), ("presctime0", _D),
    ]


class FbPlanets(C.Structure):
    _fields_ = [
        ("nb", _I),
        ("mass", _D * _NP), ("x", _D * _NP), ("y", _D * _NP),
        ("vx", _D * _NP), ("vy", _D * _NP), ("acc", _D * _NP),
        ("initial_mass", _D * _NP), ("final_mass", _D * _NP),
        ("feeldisk", _I * _NP), ("feelothers", _I * _NP), ("binary", _I * _NP),
    ]


class FbState(C.Structure):
    _fields_ = [
        ("dens", _P), ("vrad", _P), ("vtheta", _P), ("energy", _P),
        ("physical_time", _D), ("physical_time_initial", _D),
        ("omega_frame", _D), ("lost_mass", _D), ("mindt", _D), ("maxdt", _D),
        ("stardiscbarycenter_x", _D * 3), ("stardiscbarycenter_y", _D * 3),
        ("planets", FbPlanets),
    ]


class FbProfiles(C.Structure):
    _fields_ = [
        ("sigma_med", _P), ("sigma_inf", _P), ("energy_med", _P), ("vtheta_med", _P),
        ("vrad_med", _P), ("global_soundspeed", _P),
    ]


class FbDustState(C.Structure):
    _fields_ = [
        ("n", _I), ("r", _P), ("th", _P), ("vr", _P), ("vth", _P), ("l", _P), ("size", _P), ("stokes", _P),
        ("rng_x", C.c_ulonglong), ("kicks", C.c_longlong), ("carry", _D * 2), ("particles_mass", _D),
    ]


class FbTuning(C.Structure):
    _fields_ = [("cell_block", _I), ("azi_cells_per_thread", _I), ("rad_columns", _I), ("rad_rings", _I),
                ("azi_variant", _I)]


class FbStepReport(C.Structure):
    _fields_ = [
        ("substeps", _I), ("status", _I), ("physical_time", _D), ("mindt", _D), ("maxdt", _D),
        ("lost_mass", _D), ("gpu_ms", _D), ("crashes", _I), ("crash_substeps", _I),
        ("neg_density_substeps", _I), ("crash_time", _D), ("disk_on_primary", _D * 2),
        ("disk_on_primary_alt", _D * 2),
    ]


_HERE = os.path.dirname(os.path.abspath(__file__))
#: the two builds of the library (same C ABI): "parity" divides exactly and
#: rounds every multiply-add twice like the reference's build; "fast" fuses
#: multiply-adds and takes the van Leer slopes through a refined approximate
#: reciprocal
LIB_PATHS = {"parity": os.path.join(_HERE, "libfargo_b200.so"),
             "fast": os.path.join(_HERE, "libfargo_b200_fast.so")}
LIB_PATH = LIB_PATHS["parity"]


def default_mode():
    """The build used when none is named: FB_MODE from the environment, else parity."""
    mode = os.environ.get("FB_MODE", "parity")
    if mode not in LIB_PATHS:
        raise ValueError("FB_MODE must be one of %s, not %r" % (sorted(LIB_PATHS), mode))
    return mode

#: every symbol include/fargo_b200.h declares
EXPORTS = (
    "fb_params_default", "fb_params_read_par", "fb_unsupported_name", "fb_planets_read_cfg",
    "fb_init_state", "fb_create", "fb_destroy", "fb_upload", "fb_algogas", "fb_download",
    "fb_download_derived", "fb_download_crash", "fb_download_sgacc", "fb_diagnostics", "fb_planet_force", "fb_strerror", "fb_last_error", "fb_stage",
    "fb_build_info", "fb_struct_size", "fb_kernel_launches", "fb_profile", "fb_profile_read",
    "fb_select_device", "fb_transport_noalloc", "fb_noalloc_last_error", "fb_init_dust",
    "fb_dust_upload", "fb_dust_download", "fb_vortensity", "fb_batch_create", "fb_batch_algogas",
    "fb_batch_destroy", "fb_get_tuning", "fb_set_tuning", "fb_tune",
    "fb_closure_create", "fb_closure_destroy", "fb_closure_num_params", "fb_closure_params",
    "fb_closure_scales", "fb_closure_autoscale", "fb_closure_record", "fb_closure_set_sample",
    "fb_closure_loss_grad", "fb_closure_train", "fb_closure_infer", "fb_closure_apply", "fb_downsample",
    "fb_closure_set_gain", "fb_lsa_stream", "fb_rand48_state",
)

_lib = None   # the first library loaded (error details for contexts without a known library)
_libs = {}


def load(mode=None):
    """Load the library of `mode` ("parity" or "fast"; default_mode() when
    None), built by `make -C dustyfargoadsg_b200`."""
    global _lib
    mode = mode or default_mode()
    if mode in _libs:
        return _libs[mode]
    path = LIB_PATHS[mode]
    if not os.path.exists(path):
        raise RuntimeError(
            "%s is not built; run `make -C dustyfargoadsg_b200` or __graft_entry__.build()" % path)
    lib = C.CDLL(path)
    vp = C.c_void_p
    sig = {
        "fb_params_default": (_I, [C.POINTER(FbParams)]),
        "fb_params_read_par": (_I, [C.POINTER(FbParams), C.c_char_p]),
        "fb_unsupported_name": (C.c_char_p, [C.POINTER(FbParams)]),
        "fb_planets_read_cfg": (_I, [C.POINTER(FbParams), C.c_char_p, C.POINTER(FbPlanets)]),
        "fb_init_state": (_I, [C.POINTER(FbParams), vp, _D, C.c_long, C.POINTER(FbState), C.POINTER(FbProfiles)]),
        "fb_create": (_I, [C.POINTER(FbParams), _P, C.POINTER(vp)]),
        "fb_destroy": (_I, [vp]),
        "fb_upload": (_I, [vp, C.POINTER(FbState), C.POINTER(FbProfiles)]),
        "fb_algogas": (_I, [vp, C.POINTER(FbStepReport)]),
        "fb_download": (_I, [vp, C.POINTER(FbState), C.c_uint]),
        "fb_download_derived": (_I, [vp, _I, _P]),
        "fb_diagnostics": (_I, [vp, _P, _P]),
        "fb_planet_force": (_I, [vp, _D, _D, _D, _D, _P]),
        "fb_download_sgacc": (_I, [vp, _I, _I, _P, _P]),
        "fb_download_crash": (_I, [vp, C.POINTER(FbState), _P]),
        "fb_strerror": (C.c_char_p, [_I]),
        "fb_last_error": (C.c_char_p, [vp]),
        "fb_stage": (_I, [vp, _I, _D]),
        "fb_build_info": (C.c_char_p, []),
        "fb_struct_size": (_I, [_I]),
        "fb_kernel_launches": (C.c_longlong, [vp]),
        "fb_profile": (_I, [vp, _I]),
        "fb_profile_read": (_I, [vp, _I, C.POINTER(C.c_char_p), _P, C.POINTER(C.c_longlong)]),
        "fb_select_device": (_I, [_I]),
        "fb_transport_noalloc": (_I, [C.POINTER(FbParams), vp, vp, vp, vp, _D, vp, _P]),
        "fb_noalloc_last_error": (C.c_char_p, []),
        "fb_init_dust": (_I, [C.POINTER(FbParams), vp, C.c_long, C.POINTER(FbDustState)]),
        "fb_dust_upload": (_I, [vp, C.POINTER(FbDustState)]),
        "fb_dust_download": (_I, [vp, C.POINTER(FbDustState)]),
        "fb_vortensity": (_I, [vp, _P, _P, _P]),
        "fb_batch_create": (_I, [C.POINTER(vp), _I, C.POINTER(vp)]),
        "fb_batch_algogas": (_I, [vp, C.POINTER(FbStepReport)]),
        "fb_batch_destroy": (_I, [vp]),
        "fb_get_tuning": (_I, [vp, C.POINTER(FbTuning)]),
        "fb_set_tuning": (_I, [vp, C.POINTER(FbTuning)]),
        "fb_tune": (_I, [vp, _I, C.POINTER(FbTuning), C.POINTER(_D)]),
        "fb_closure_create": (_I, [vp, _I, _I, C.c_ulonglong, C.POINTER(vp)]),
        "fb_closure_destroy": (_I, [vp]),
        "fb_closure_num_params": (_I, [vp, C.POINTER(_I), C.POINTER(_I)]),
        "fb_closure_params": (_I, [vp, _FP, _FP, _I]),
        "fb_closure_scales": (_I, [vp, _P, _P, _I]),
        "fb_closure_autoscale": (_I, [vp, _I]),
        "fb_closure_record": (_I, [vp, vp, _I, _I]),
        "fb_closure_set_sample": (_I, [vp, _I, _FP, _FP, _FP]),
        "fb_closure_loss_grad": (_I, [vp, _I, _I, C.POINTER(_D), _FP, _FP]),
        "fb_closure_train": (_I, [vp, _I, _I, _I, _I, _D, C.c_ulonglong, _P]),
        "fb_closure_infer": (_I, [vp, vp, _I, _FP]),
        "fb_closure_apply": (_I, [vp, vp]),
        "fb_downsample": (_I, [vp, vp]),
        "fb_closure_set_gain": (_I, [vp, _D]),
        "fb_lsa_stream": (_I, [vp, C.POINTER(C.c_ulonglong), _I]),
        "fb_rand48_state": (C.c_ulonglong, [C.c_long, C.c_longlong]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    check_layout(lib)
    lib.fb_mode = mode
    _libs[mode] = lib
    if _lib is None:
        _lib = lib
    return lib


def check_layout(lib):
    for idx, cls in enumerate((FbParams, FbPlanets, FbState, FbProfiles, FbStepReport, FbDustState, FbTuning)):
        want = lib.fb_struct_size(idx)
        if want != C.sizeof(cls):
            raise RuntimeError("ABI mismatch for %s: C %d bytes, ctypes %d" % (cls.__name__, want, C.sizeof(cls)))


class FbError(RuntimeError):
    def __init__(self, code, where, detail=""):
        self.code = code
        name = FB_ERR.get(code, str(code))
        super().__init__("%s failed: %s%s" % (where, name, (" (" + detail + ")") if detail else ""))


def check(code, where, ctx=None, lib=None):
    if code != FB_OK:
        detail = ""
        lib = lib or _lib
        if ctx is not None and lib is not None:
            detail = (lib.fb_last_error(ctx) or b"").decode(errors="replace")
        raise FbError(code, where, detail)
