"""ctypes binding of libalfa.so (the C-ABI declared in include/alfa.h).

The library is loaded from this package directory only; there is no CPU
fallback: without a built library or without a CUDA device every entry point
raises."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libalfa.so")

c_double_p = ctypes.POINTER(ctypes.c_double)
c_void_p = ctypes.c_void_p


class AlfaConfig(ctypes.Structure):
    """``alfa_config`` (include/alfa.h); field names are the reference's
    Config.py option names."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("l_x", ctypes.c_double), ("l_y", ctypes.c_double), ("l_z", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("istep", ctypes.c_int),
        ("Ugal", ctypes.c_double),
        ("optSurfFlux", ctypes.c_int), ("optSurfBC", ctypes.c_int),
        ("z0m", ctypes.c_double), ("z0T", ctypes.c_double), ("zTemperature", ctypes.c_double),
        ("SensibleHeatFlux", ctypes.c_double),
        ("Ug2", ctypes.c_double), ("Vg2", ctypes.c_double),
        ("f_coriolis", ctypes.c_double),
        ("inversion", ctypes.c_double),
        ("optBuoyancy", ctypes.c_int),
        ("T_0", ctypes.c_double),
        ("optSgs", ctypes.c_int), ("dynamicSGS_call_time", ctypes.c_int), ("FGR", ctypes.c_int),
        ("Cs2", ctypes.c_double), ("Cs2PrRatio", ctypes.c_double),
        ("optDamping", ctypes.c_int),
        ("z_damping", ctypes.c_double), ("RelaxTime", ctypes.c_double),
        ("optAdvection", ctypes.c_int),
        ("optPressureSolver", ctypes.c_int),
        ("optGeoWind", ctypes.c_int),
        ("optMoisture", ctypes.c_int), ("optMoistureSurfBC", ctypes.c_int),
        ("MoistureFlux", ctypes.c_double), ("zMoisture", ctypes.c_double),
        ("q_inversion", ctypes.c_double),
        ("precision", ctypes.c_int),
    ]


# alfa_config.precision
FP64, FP32, MIXED = 0, 1, 2


class AlfaDerived(ctypes.Structure):
    _fields_ = [
        ("mx", ctypes.c_int), ("my", ctypes.c_int), ("nx_rfft", ctypes.c_int),
        ("ny_rfft", ctypes.c_int),
        ("z_scale", ctypes.c_double), ("g_nondim", ctypes.c_double),
        ("f_coriolis_nondim", ctypes.c_double), ("T_0_nondim", ctypes.c_double),
        ("inversion_nondim", ctypes.c_double),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("L", ctypes.c_double), ("dt_nondim", ctypes.c_double), ("TFR", ctypes.c_double),
        ("cut_explicit", ctypes.c_int * 2), ("cut_level1", ctypes.c_int * 2),
        ("cut_level2", ctypes.c_int * 2),
    ]


class AlfaDiag(ctypes.Structure):
    _fields_ = [("iteration", ctypes.c_int), ("CFL", ctypes.c_double), ("CFLmax", ctypes.c_double),
                ("ustar_rms", ctypes.c_double), ("qz_sfc_avg", ctypes.c_double)]


P = c_void_p          # device pointer
PP = ctypes.POINTER(c_void_p)  # array of device pointers
CTX = c_void_p
I = ctypes.c_int
D = ctypes.c_double

# name -> argument types (after the context); every function returns int
SIGNATURES = {
    "alfa_FFT": [P, P],
    "alfa_FFT_pad": [P, P],
    "alfa_Dealias1": [P, P],
    "alfa_Dealias2": [P, P],
    "alfa_Filtering_Explicit": [P, P, P],
    "alfa_Filtering_Level1": [P, P],
    "alfa_Filtering_Level2": [P, P],
    "alfa_Derivxy": [P, I, P],
    "alfa_velocityGradients": [P, P, P, P, P, P, P, P, P, PP],
    "alfa_potentialTemperatureGradients": [P, P, P, P, PP],
    "alfa_moistureGradients": [P, P, P, P, PP],
    "alfa_SurfaceMoistureFlux_HomogeneousPrescribedQ": [P, P, D, PP, P],
    "alfa_SurfaceMoistureFlux_HeterogeneousPrescribedQ": [P, P, D, PP, P],
    "alfa_Derivz_Generic_uvp": [P, P],
    "alfa_Derivz_Generic_w": [P, P],
    "alfa_PlanarMean": [P, P],
    "alfa_Imfilter": [P, P],
    "alfa_ComputeBeta": [P, I, P],
    "alfa_SurfaceFlux_HomogeneousConstantFlux": [P, P, P, PP, P, P, P, P, PP],
    "alfa_SurfaceFlux_HeterogeneousConstantFlux": [P, P, P, PP, P, P, P, P, PP],
    "alfa_SurfaceFlux_HomogeneousVaryingFlux": [P, P, P, D, PP, P, P, P, P, P, PP],
    "alfa_SurfaceFlux_HeterogeneousVaryingFlux": [P, P, P, D, PP, P, P, P, P, P, PP],
    "alfa_SurfaceFlux_HomogeneousPrescribedTemperature": [P, P, P, D, PP, P, P, P, P, P, PP],
    "alfa_SurfaceFlux_HeterogeneousPrescribedTemperature": [P, P, P, D, PP, P, P, P, P, P, PP],
    "alfa_Advection": [P] * 12,
    "alfa_ScalarAdvection": [P] * 7,
    "alfa_BuoyancyOpt1": [P, P, P],
    "alfa_BuoyancyOpt2": [P, P, P],
    "alfa_DivStressDynamicSGS": [PP, P, P, P, P, P, P, P, P, P, P, P, P, P, PP],
    "alfa_DivFluxDynamicSGS": [PP, P, P, P, P, P, P, P, P, P, P],
    "alfa_DivStressStaticSGS": [PP, P, P, P, P, P, P, P, P, P, PP],
    "alfa_DivFluxStaticSGS": [PP, P, P, P, P, P, P, P],
    "alfa_RHS_Momentum": [P] * 17,
    "alfa_RHS_Scalar": [P] * 5,
    "alfa_RHS_Moisture": [P] * 5,
    "alfa_PressureRC": [P] * 13,
    "alfa_ThomasPressureSolve": [P] * 7,
    "alfa_AB2_uvw": [P] * 12,
    "alfa_AB2_TH": [P] * 4,
    "alfa_AB2_Q": [P] * 4,
    "alfa_AddPressureGradient": [P] * 6,
    "alfa_CFL": [P] * 4,
    "alfa_init_state": [P] * 4,
    "alfa_set_series": [c_double_p, c_double_p, c_double_p, c_double_p, I],
    "alfa_set_geowind_series": [c_double_p, c_double_p, I],
    "alfa_init_moisture": [P],
    "alfa_set_moisture_series": [c_double_p, c_double_p, I],
    "alfa_get_moisture": [P],
    "alfa_step": [I],
    "alfa_get_state": [P] * 5,
    "alfa_ComputeStats": [P] * 24,
    "alfa_stats_sample": [P],
    "alfa_save_checkpoint": [P],
    "alfa_load_checkpoint": [P],
    "alfa_step_graph": [I],
}

class AlfaTuneEntry(ctypes.Structure):
    """``alfa_tune_entry`` (include/alfa.h)."""
    _fields_ = [("axis", ctypes.c_int), ("n_in", ctypes.c_int), ("n_out", ctypes.c_int),
                ("outputs", ctypes.c_int), ("map", ctypes.c_int), ("variant", ctypes.c_int),
                ("chosen", ctypes.c_int), ("equal", ctypes.c_int), ("ms", ctypes.c_double)]


class AlfaMlpReport(ctypes.Structure):
    _fields_ = [("steps", I), ("learned_steps", I), ("judged", I), ("reverted", I),
                ("reverted_at", I), ("last_drift", D), ("max_drift", D),
                ("window_drift", D), ("max_window_drift", D)]


_lib = None


class AlfaError(RuntimeError):
    pass


def load():
    """Load libalfa.so (built by ``jax_alfa_b200.build``); raise if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AlfaError(f"{LIB_PATH} is missing: run `python -m jax_alfa_b200.build` "
                        "(the CUDA library is required; there is no CPU path)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.alfa_create.argtypes = [ctypes.POINTER(AlfaConfig), ctypes.POINTER(c_void_p)]
    lib.alfa_create.restype = I
    lib.alfa_destroy.argtypes = [CTX]
    lib.alfa_destroy.restype = None
    lib.alfa_last_error.argtypes = [CTX]
    lib.alfa_last_error.restype = ctypes.c_char_p
    lib.alfa_set_stream.argtypes = [CTX, c_void_p]
    lib.alfa_set_stream.restype = I
    lib.alfa_get_derived.argtypes = [CTX, ctypes.POINTER(AlfaDerived)]
    lib.alfa_get_derived.restype = I
    lib.alfa_get_precision.argtypes = [CTX]
    lib.alfa_get_precision.restype = I
    lib.alfa_workspace_bytes.argtypes = [CTX]
    lib.alfa_workspace_bytes.restype = ctypes.c_size_t
    lib.alfa_get_diag.argtypes = [CTX, ctypes.POINTER(AlfaDiag)]
    lib.alfa_get_diag.restype = I
    lib.alfa_launch_count.argtypes = []
    lib.alfa_launch_count.restype = ctypes.c_ulonglong
    lib.alfa_time_kernel.argtypes = [CTX, I, I, c_double_p, c_double_p]
    lib.alfa_time_kernel.restype = I
    lib.alfa_autotune.argtypes = [CTX, I, ctypes.POINTER(AlfaTuneEntry), I,
                                  ctypes.POINTER(ctypes.c_int)]
    lib.alfa_autotune.restype = I
    lib.alfa_set_line_variant.argtypes = [CTX, I, I, I, I, I, I]
    lib.alfa_set_line_variant.restype = I
    lib.alfa_tc_line_apply.argtypes = [CTX, I, I, I, I, D, ctypes.c_longlong, P, P]
    lib.alfa_tc_line_apply.restype = I
    lib.alfa_set_tc_spin_limit.argtypes = [CTX, ctypes.c_ulonglong]
    lib.alfa_set_tc_spin_limit.restype = I
    lib.alfa_PlanarMean_noalloc.argtypes = [P, I, I, I, P, c_void_p]
    lib.alfa_PlanarMean_noalloc.restype = I
    lib.alfa_checkpoint_doubles.argtypes = [CTX]
    lib.alfa_checkpoint_doubles.restype = ctypes.c_size_t
    lib.alfa_ensemble_create.argtypes = [ctypes.POINTER(c_void_p), I, ctypes.POINTER(c_void_p)]
    lib.alfa_ensemble_create.restype = I
    lib.alfa_ensemble_step.argtypes = [c_void_p, I]
    lib.alfa_ensemble_step.restype = I
    lib.alfa_ensemble_sync.argtypes = [c_void_p]
    lib.alfa_ensemble_sync.restype = I
    lib.alfa_ensemble_set_stream.argtypes = [c_void_p, c_void_p]
    lib.alfa_ensemble_set_stream.restype = I
    lib.alfa_ensemble_error.argtypes = [c_void_p]
    lib.alfa_ensemble_error.restype = ctypes.c_char_p
    lib.alfa_ensemble_destroy.argtypes = [c_void_p]
    lib.alfa_ensemble_destroy.restype = None
    M = c_void_p
    for name, args in {
            "alfa_mlp_create": [CTX, I, ctypes.c_ulonglong, ctypes.POINTER(c_void_p)],
            "alfa_mlp_collect": [M, I],
            "alfa_mlp_train": [M, I, I, D, c_double_p],
            "alfa_mlp_loss_grad": [M, P, P, P, I, P, P],
            "alfa_mlp_get_params": [M, P, P],
            "alfa_mlp_set_params": [M, P, P],
            "alfa_mlp_features": [M, P],
            "alfa_mlp_infer": [M, P, P],
            "alfa_step_learned": [M, I, I, D, I, I, ctypes.POINTER(AlfaMlpReport)]}.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = I
    lib.alfa_mlp_destroy.argtypes = [M]
    lib.alfa_mlp_destroy.restype = None
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = [CTX] + args
        f.restype = I
    _lib = lib
    return lib


def exported_symbols():
    """Names the header declares (parsed from include/alfa.h)."""
    import re
    hdr = os.path.join(os.path.dirname(HERE), "include", "alfa.h")
    with open(hdr) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(alfa_[A-Za-z0-9_]+)\s*\(", text)))
