"""Loader of ``libymgpu.so`` (the engine's CUDA kernels behind a C ABI).

The library is built in-tree (``yang-mills_b200/lib/libymgpu.so``) by
``yang-mills_b200/csrc/Makefile``.  There is no CPU fallback: if the library
is missing or no CUDA device answers, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_PKG), "lib", "libymgpu.so")

i32, i64, u64, f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_double
P = C.POINTER
VP = C.c_void_p


class EnsembleDesc(C.Structure):
    _fields_ = [("group", i32), ("precision", i32), ("n_chains", i64), ("extents", P(i64)),
                ("beta", P(f64)), ("chain_seed", P(u64)), ("lift_reference_caps", i32),
                ("device", i32)]


class MeasuredRun(C.Structure):
    _fields_ = [("proposal_angle", f64), ("generator_mode", i32), ("polyakov_direction", i32),
                ("n_blocks", i64), ("sweeps_per_block", i64), ("rmax", i32), ("tmax", i32)]


class GlueballPlan(C.Structure):
    _fields_ = [("rho", f64), ("n_levels", i32), ("levels", P(i64)), ("n_blocked", i32),
                ("fine", P(VP)), ("coarse", P(VP)), ("first_chain", P(i64))]


# name -> (argtypes); every function returns int32 ym_status
SIGNATURES = {
    "ym_last_cuda_error": [],
    "ym_ensemble_create": [P(EnsembleDesc), P(VP)],
    "ym_ensemble_destroy": [VP],
    "ym_ensemble_info": [VP, P(i64), P(i64), P(i32), P(i32)],
    "ym_ensemble_set_identity": [VP],
    "ym_ensemble_hot_start": [VP],
    "ym_ensemble_upload": [VP, i64, P(f64)],
    "ym_ensemble_download": [VP, i64, P(f64)],
    "ym_ensemble_set_sweep_index": [VP, u64],
    "ym_ensemble_get_sweep_index": [VP, P(u64)],
    "ym_ensemble_synchronize": [VP],
    "ym_ensemble_stream": [VP, P(VP)],
    "ym_su3_metropolis_sweeps": [VP, f64, i32, i64],
    "ym_su3_accounting": [VP, P(u64), P(u64)],
    "ym_ensemble_set_sweep_path": [VP, i32],
    "ym_ensemble_lift_angle_cap": [VP, i32],
    "ym_ensemble_set_fast_sweeps": [VP, i32],
    "ym_ensemble_get_fast_sweeps": [VP, P(i32)],
    "ym_ensemble_set_sweep_layout": [VP, i32, i32],
    "ym_ensemble_get_sweep_layout": [VP, P(i32), P(i32), P(i32)],
    "ym_ensemble_get_sweep_path": [VP, P(i32)],
    "ym_su3_measured_sweeps": [VP, f64, i32, i64, i64, P(f64)],
    "ym_su3_measured_run": [VP, VP, P(MeasuredRun), P(f64), P(f64), P(f64)],
    "ym_reset_accounting": [VP],
    "ym_su3_reference_sweeps": [VP, f64, P(u64), i64, P(u64), P(u64)],
    "ym_su3_reference_average_plaquette": [VP, P(f64)],
    "ym_average_plaquette": [VP, P(f64)],
    "ym_su3_max_residuals": [VP, P(f64), P(f64)],
    "ym_ensemble_set_chain": [VP, i64, f64, u64],
    "ym_proposal_angle_from_u64": [u64, f64, P(f64)],
    "ym_su3_average_plaquette_noalloc": [VP, P(i64), VP, VP],
    "ym_su3_wilson_loops": [VP, i32, i32, P(f64)],
    "ym_su2_wilson_loops": [VP, i32, i32, P(f64)],
    "ym_su2_polyakov_loops": [VP, i32, P(f64)],
    "ym_rectangular_path": [i32, i32, i64, i64, P(i32), i64, P(i64)],
    "ym_path_holonomy": [VP, i64, P(i64), P(i32), i64, P(f64), P(i64)],
    "ym_wilson_loop": [VP, i64, P(i64), P(i32), i64, P(f64)],
    "ym_wilson_loop_sites": [VP, i64, P(i32), i64, P(f64)],
    "ym_polyakov_loop": [VP, i64, P(i64), i32, P(f64)],
    "ym_polyakov_loop_sites": [VP, i64, i32, P(f64)],
    "ym_plaquette": [VP, i64, P(i64), i32, i32, P(f64)],
    "ym_wilson_action": [VP, f64, P(f64)],
    "ym_su2_staple": [VP, i64, P(i64), i32, P(f64), P(i64)],
    "ym_su3_local_link_action": [VP, i64, P(i64), i32, f64, P(f64)],
    "ym_su3_local_action_difference": [VP, i64, P(i64), i32, P(f64), f64, P(f64)],
    "ym_su3_gauge_transform": [VP, i64, P(f64), VP, i64],
    "ym_ensemble_get_link": [VP, i64, P(i64), i32, P(f64)],
    "ym_ensemble_set_link": [VP, i64, P(i64), i32, P(f64)],
    "ym_su3_polyakov_loops": [VP, i32, P(f64)],
    "ym_su3_scalar_operator_basis": [VP, P(f64), P(f64)],
    "ym_ensemble_copy": [VP, VP],
    "ym_ensemble_copy_chain": [VP, i64, VP, i64],
    "ym_ensemble_copy_chains": [VP, i64, VP, i64, i64],
    "ym_su3_spatial_stout_smear": [VP, VP, f64, i64, i32],
    "ym_su3_spatial_stride2_block": [VP, VP],
    "ym_su3_glueball_measure": [VP, VP, P(GlueballPlan), P(f64), P(f64), P(f64), P(f64)],
    "ym_su3_glueball_prepare": [VP, VP, P(GlueballPlan)],
    "ym_periodic_connected_estimator": [P(f64), i64, i64, P(f64), P(f64), P(f64)],
    "ym_connected_from_samples": [P(f64), i64, i64, i64, P(f64)],
    "ym_jackknife_replicas": [P(f64), i64, i64, P(f64)],
    "ym_jackknife_covariance": [P(f64), i64, i64, i64, i64, P(f64)],
    "ym_su3_reunitarize": [VP],
    "ym_ensemble_convert": [VP, VP],
    "ym_su2_markov_sweeps": [VP, i64, i64, i32, i64],
    "ym_su2_measured_sweeps": [VP, i64, i64, i32, i64, i64, P(f64)],
    "ym_su2_overrelaxation_sweeps": [VP, i64],
    "ym_su2_accounting": [VP, P(u64), P(u64)],
    "ym_su2_max_unit_residual": [VP, P(f64)],
    "ym_profile_enable": [VP, i32],
    "ym_profile_read": [VP, i32, P(f64), P(i64)],
    # learned proposal (include/ym_learned.h)
    "ym_model_create": [i32, u64, f64, P(VP)],
    "ym_model_destroy": [VP],
    "ym_device_wait_selftest": [i32, i64],
    "ym_device_release_pooled_memory": [i32],
    "ym_model_get_params": [VP, P(C.c_float)],
    "ym_model_set_params": [VP, P(C.c_float)],
    "ym_model_forward": [VP, P(C.c_float), i64, P(C.c_float)],
    "ym_model_gradient": [VP, P(C.c_float), P(C.c_float), P(f64), i64, P(f64), P(C.c_float)],
    "ym_learned_records": [VP, i32, i32, P(C.c_float), P(C.c_float), P(f64), P(i64)],
    "ym_model_train": [VP, VP, i64, i64, f64, f64, P(f64)],
    "ym_su3_learned_sweeps": [VP, VP, i64],
    "ym_su3_learned_measured_sweeps": [VP, VP, i64, i64, P(f64)],
}

KERNEL_IDS = {"su3_metropolis": 0, "plaquette": 1, "su2_heatbath": 2, "su2_overrelax": 3,
              "stout": 4, "operators": 5, "aux": 6, "learned": 7}


class ChainDiagnostics(C.Structure):
    _fields_ = [("mean", f64), ("variance", f64), ("positive_window_lag", i64),
                ("integrated_autocorrelation_time", f64), ("effective_sample_size", f64),
                ("standard_error", f64)]


class EfficiencyReport(C.Structure):
    _fields_ = [("diagnostics", ChainDiagnostics), ("reweighting_efficiency", f64),
                ("weight_only_ess", f64), ("combined_ess_proxy", f64), ("total_cost", f64),
                ("sampling_cost_per_effective_sample_proxy", f64),
                ("total_cost_per_effective_sample_proxy", f64)]


SIGNATURES.update({
    "ym_diagnostics": [P(f64), i64, i64, P(ChainDiagnostics), P(f64)],
    "ym_sampling_efficiency": [P(f64), i64, P(f64), i64, f64, f64, f64, P(EfficiencyReport),
                               P(f64)],
})


# host analysis (include/ym_analysis.h)
class EffectiveMassPoint(C.Structure):
    _fields_ = [("tau", i64), ("full_estimate", f64), ("jackknife_mean", f64),
                ("standard_error", f64)]


class FitWindowC(C.Structure):
    _fields_ = [("start", u64), ("end", u64)]


class ScalarFitResultC(C.Structure):
    _fields_ = [("time_extent", i64), ("jackknife_replicates", i64), ("selected_window", FitWindowC),
                ("plateau_weighted_effective_mass", f64), ("plateau_maximum_z", f64),
                ("fitted_mass", f64), ("fitted_amplitude", f64), ("chi_square", f64),
                ("degrees_of_freedom", i64), ("chi_square_per_dof", f64),
                ("mass_jackknife_mean", f64), ("mass_standard_error", f64),
                ("amplitude_jackknife_mean", f64), ("amplitude_standard_error", f64),
                ("maximum_off_diagonal_correlation", f64)]


class PrincipalProjectionC(C.Structure):
    _fields_ = [("reference_time", i64), ("diagonalization_time", i64),
                ("principal_eigenvalue", f64), ("coefficients", f64 * 2)]


SIGNATURES.update({
    "ym_cosh_effective_mass_with_jackknife": [P(f64), i64, P(P(f64)), P(i64), i64, P(u64), i64,
                                              P(EffectiveMassPoint)],
    "ym_analytic_periodic_single_state": [i64, f64, f64, P(f64)],
    "ym_correlated_scalar_fit": [P(f64), i64, P(P(f64)), P(i64), i64, P(FitWindowC), i64,
                                 P(ScalarFitResultC)],
    "ym_scalar_fit_window_covariance": [P(P(f64)), P(i64), i64, FitWindowC, P(f64)],
    "ym_scalar_fit_invert_covariance": [P(f64), i64, P(f64)],
    "ym_maximum_off_diagonal_correlation": [P(f64), i64, P(f64)],
    "ym_canonical_scalar_fit_fixture": [P(f64), P(f64), P(FitWindowC)],
    "ym_scalar_variational_connected_correlator": [P(f64), i64, i64, P(f64), P(f64)],
    "ym_principal_generalized_projection": [P(f64), i64, i64, i64, P(PrincipalProjectionC), P(f64)],
    "ym_canonical_two_state_matrices": [P(f64)],
    "ym_max_matrix_series_residual": [P(f64), i64, P(f64), i64, P(f64)],
})
SIGNATURES.update({
    # canonical configurations (include/ym_config.h)
    "ym_su2_to_canonical_config": [P(i64), P(f64), i32, C.c_char_p, i64, P(i64)],
    "ym_su2_from_canonical_config": [C.c_char_p, i64, i32, P(i64), P(f64), i64],
    "ym_su3_to_canonical_config": [P(i64), P(f64), i32, C.c_char_p, i64, P(i64)],
    "ym_su3_from_canonical_config": [C.c_char_p, i64, i32, P(i64), P(f64), i64],
})
U64_FUNCTIONS = {
    "ym_derive_chain_seed": [u64, u64],
    "ym_derive_su3_chain_seed": [u64, u64],
    "ym_splitmix64_at": [u64, u64],
}

_lib = None


def lib() -> C.CDLL:
    """Load libymgpu.so once; raise loudly when it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libymgpu.so not built at {LIB_PATH}; run `make -C yang-mills_b200/csrc` "
                "(the engine has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, argtypes in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = argtypes
            fn.restype = i32
        for name, argtypes in U64_FUNCTIONS.items():
            fn = getattr(L, name)
            fn.argtypes = argtypes
            fn.restype = u64
        _lib = L
    return _lib
