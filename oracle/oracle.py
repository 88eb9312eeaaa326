"""ctypes loader for the CPU oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference crate
(QSOLKCB/YANG-MILLS, ``reference/rust/src``) in plain C; this module exposes
it to the test-suite, to ``__graft_entry__.smoke()`` and to the CPU-baseline
leg of ``bench.py`` as the checker.  The product (``yang-mills_b200``) never
imports it.

Lattices are numpy arrays in the reference's memory order: SU(3) as
``(links, 3, 3)`` complex128, SU(2) as ``(links, 4)`` float64, link index
``site*4 + mu`` with lexicographic sites (x3 fastest).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

i64 = C.c_int64
u64 = C.c_uint64
f64 = C.c_double
P = C.POINTER


class OracleError(RuntimeError):
    """A nonzero ym_status returned by the oracle."""

    def __init__(self, code: int, what: str):
        super().__init__(f"{what} failed with ym_status {code}")
        self.code = code


class Su3Config(C.Structure):
    _fields_ = [("extents", i64 * 4), ("beta", f64), ("master_seed", u64), ("chain_id", u64),
                ("thermalization_sweeps", i64), ("measurements", i64),
                ("sweeps_between_measurements", i64), ("proposal_angle", f64),
                ("autocorrelation_max_lag", i64)]


class Su3Scalars(C.Structure):
    _fields_ = [("derived_seed", u64), ("total_sweeps", i64), ("proposals", u64),
                ("accepts", u64), ("mean_acceptance", f64),
                ("final_unitarity_residual", f64), ("final_determinant_residual", f64)]


class Su2Config(C.Structure):
    _fields_ = [("extents", i64 * 4), ("beta", f64), ("master_seed", u64), ("chain_id", u64),
                ("thermalization_sweeps", i64), ("measurements", i64),
                ("sweeps_between_measurements", i64),
                ("overrelaxation_sweeps_per_heatbath", i64),
                ("max_heatbath_attempts_per_link", i64), ("autocorrelation_max_lag", i64)]


class Su2Scalars(C.Structure):
    _fields_ = [("derived_seed", u64), ("total_heatbath_sweeps", i64),
                ("total_overrelaxation_sweeps", i64), ("heatbath_proposals", u64),
                ("heatbath_updates", u64), ("mean_heatbath_acceptance", f64),
                ("final_link_unit_residual", f64)]


class Diagnostics(C.Structure):
    _fields_ = [("mean", f64), ("variance", f64), ("positive_window_lag", i64),
                ("integrated_autocorrelation_time", f64), ("effective_sample_size", f64),
                ("standard_error", f64)]


class Efficiency(C.Structure):
    _fields_ = [("diagnostics", Diagnostics), ("reweighting_efficiency", f64),
                ("weight_only_ess", f64), ("combined_ess_proxy", f64), ("total_cost", f64),
                ("sampling_cost_per_effective_sample_proxy", f64),
                ("total_cost_per_effective_sample_proxy", f64)]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, no FMA)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.or_mix64_pub.restype = u64
        L.or_mix64_pub.argtypes = [u64]
        L.or_splitmix_next.restype = u64
        L.or_splitmix_next.argtypes = [P(u64)]
        L.or_splitmix_unit.restype = f64
        L.or_splitmix_unit.argtypes = [P(u64)]
        for name in ("or_derive_chain_seed", "or_derive_su3_chain_seed", "or_splitmix_at"):
            getattr(L, name).restype = u64
            getattr(L, name).argtypes = [u64, u64]
        L.or_cb_link_key.restype = u64
        L.or_cb_link_key.argtypes = [u64, u64, i64, C.c_int]
        L.or_proposal_angle_from_u64.argtypes = [u64, f64, P(f64)]
        L.or_su3_cb_sweep.argtypes = [P(i64), P(f64), f64, f64, u64, u64, C.c_int, P(u64), P(u64)]
        L.or_su3_metropolis_sweep.argtypes = [P(i64), P(f64), f64, f64, P(u64), P(u64), P(u64)]
        L.or_su2_heatbath_sweep.argtypes = [P(i64), P(f64), f64, P(u64), i64, P(u64), P(u64)]
        L.or_su2_sample_heatbath.argtypes = [f64, P(u64), i64, P(f64), P(u64)]
        L.or_sampling_efficiency.argtypes = [P(f64), i64, P(f64), i64, f64, f64, f64,
                                             P(Efficiency), P(f64)]
        L.or_su3_generator_rotation.argtypes = [C.c_int, f64, P(f64)]
        L.or_su3_visit.argtypes = [P(f64), P(f64), f64, f64, u64, C.c_int, P(u64)]
        L.or_bench_su3_reference.argtypes = [P(i64), f64, f64, u64, i64, i64, P(f64), P(u64)]
        L.or_su2_from_axis_angle.argtypes = [P(f64), f64, P(f64)]
        L.or_su2_wilson_action.argtypes = [P(i64), P(f64), f64, P(f64)]
        L.or_su3_wilson_action.argtypes = [P(i64), P(f64), f64, P(f64)]
        L.or_su3_local_action_difference.argtypes = [P(i64), P(f64), P(i64), C.c_int, P(f64),
                                                     f64, P(f64)]
        L.or_spatial_stout_smear.argtypes = [P(i64), P(f64), f64, i64, C.c_int, P(f64)]
        L.or_jackknife_covariance.argtypes = [P(f64), i64, i64, i64, i64, P(f64)]
        L.or_connected_from_samples.argtypes = [P(f64), i64, i64, i64, P(f64)]
        L.or_periodic_connected_estimator.argtypes = [P(f64), i64, i64, P(f64), P(f64), P(f64)]
        L.or_diagnostics.argtypes = [P(f64), i64, i64, P(Diagnostics), P(f64)]
        L.or_scalar_a1pp_operator_basis.argtypes = [P(i64), P(f64), i64, P(f64), P(f64),
                                                    P(i64), P(i64)]
        L.or_scalar_connected_correlators.argtypes = [P(i64), P(f64), i64, P(f64), P(f64),
                                                      P(f64)]
        _lib = L
    return _lib


# ---------------------------------------------------------------- helpers

def _check(code: int, what: str) -> None:
    if code != 0:
        raise OracleError(code, what)


def _ext(extents) -> C.Array:
    return (i64 * 4)(*[int(v) for v in extents])


def _x(x) -> C.Array:
    return (i64 * 4)(*[int(v) for v in x])


def _dp(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(P(f64))


def su3_links(n_links: int) -> np.ndarray:
    return np.zeros((n_links, 3, 3), dtype=np.complex128)


def n_links(extents) -> int:
    return int(np.prod(extents)) * 4


def site_index(extents, x) -> int:
    return ((x[0] * extents[1] + x[1]) * extents[2] + x[2]) * extents[3] + x[3]


# ---------------------------------------------------------------- RNG / seeds

def mix64(v: int) -> int:
    return lib().or_mix64_pub(v)


def splitmix_outputs(seed: int, n: int) -> list:
    s = u64(seed)
    return [lib().or_splitmix_next(C.byref(s)) for _ in range(n)]


def derive_chain_seed(master: int, chain: int) -> int:
    return lib().or_derive_chain_seed(master, chain)


def derive_su3_chain_seed(master: int, chain: int) -> int:
    return lib().or_derive_su3_chain_seed(master, chain)


def splitmix_at(seed: int, n: int) -> int:
    return lib().or_splitmix_at(seed, n)


def cb_link_key(chain_seed: int, sweep: int, lex: int, mu: int) -> int:
    return lib().or_cb_link_key(chain_seed, sweep, lex, mu)


def proposal_angle_from_u64(raw: int, angle: float) -> float:
    out = f64()
    _check(lib().or_proposal_angle_from_u64(raw, angle, C.byref(out)), "proposal_angle_from_u64")
    return out.value


# ---------------------------------------------------------------- SU(3)

def su3_identity(extents, lift_cap: bool = False) -> np.ndarray:
    links = su3_links(n_links(extents))
    links[:] = np.eye(3)
    if not lift_cap and n_links(extents) > (1 << 18):
        raise OracleError(7, "su3_identity")
    return links


def su3_from_algebra(coef) -> np.ndarray:
    c = np.ascontiguousarray(coef, dtype=np.float64)
    out = np.zeros((3, 3), np.complex128)
    _check(lib().or_su3_from_algebra(_dp(c), _dp(out.view(np.float64))), "from_algebra")
    return out


def su3_generator_rotation(g: int, theta: float) -> np.ndarray:
    out = np.zeros((3, 3), np.complex128)
    _check(lib().or_su3_generator_rotation(g, theta, _dp(out.view(np.float64))), "rotation")
    return out


def su3_traceless_cycle_link() -> np.ndarray:
    out = np.zeros((3, 3), np.complex128)
    _check(lib().or_su3_traceless_cycle_link(_dp(out.view(np.float64))), "cycle link")
    return out


def su3_deterministic_site_gauge(x) -> np.ndarray:
    out = np.zeros((3, 3), np.complex128)
    _check(lib().or_su3_deterministic_site_gauge(_x(x), _dp(out.view(np.float64))), "gauge")
    return out


def su3_gauge_transform(extents, links: np.ndarray, site_gauges: np.ndarray) -> np.ndarray:
    out = np.empty_like(links)
    _check(lib().or_su3_gauge_transform(_ext(extents), _dp(links.view(np.float64)),
                                        _dp(site_gauges.view(np.float64)),
                                        _dp(out.view(np.float64))), "gauge_transform")
    return out


def su3_deterministic_gauge_field(extents) -> np.ndarray:
    g = np.zeros((int(np.prod(extents)), 3, 3), np.complex128)
    for x0 in range(extents[0]):
        for x1 in range(extents[1]):
            for x2 in range(extents[2]):
                for x3 in range(extents[3]):
                    g[site_index(extents, (x0, x1, x2, x3))] = su3_deterministic_site_gauge(
                        (x0, x1, x2, x3))
    return g


def su3_average_plaquette(extents, links: np.ndarray) -> float:
    out = f64()
    _check(lib().or_su3_average_plaquette(_ext(extents), _dp(links.view(np.float64)),
                                          C.byref(out)), "average_plaquette")
    return out.value


def su3_plaquette_value(extents, links, x, mu, nu) -> float:
    out = f64()
    _check(lib().or_su3_plaquette_value(_ext(extents), _dp(links.view(np.float64)), _x(x), mu,
                                        nu, C.byref(out)), "plaquette_value")
    return out.value


def su3_wilson_action(extents, links, beta) -> float:
    out = f64()
    _check(lib().or_su3_wilson_action(_ext(extents), _dp(links.view(np.float64)), beta,
                                      C.byref(out)), "wilson_action")
    return out.value


def su3_max_residuals(extents, links):
    u, d = f64(), f64()
    _check(lib().or_su3_max_residuals(_ext(extents), _dp(links.view(np.float64)), C.byref(u),
                                      C.byref(d)), "max_residuals")
    return u.value, d.value


def su3_polyakov_loop(extents, links, start, direction) -> complex:
    re, im = f64(), f64()
    _check(lib().or_su3_polyakov_loop(_ext(extents), _dp(links.view(np.float64)), _x(start),
                                      direction, C.byref(re), C.byref(im)), "polyakov_loop")
    return complex(re.value, im.value)


def su3_plaquette_matrix(extents, links, x, mu, nu) -> np.ndarray:
    out = np.zeros((3, 3), np.complex128)
    _check(lib().or_su3_plaquette_matrix(_ext(extents), _dp(links.view(np.float64)), _x(x), mu,
                                         nu, _dp(out.view(np.float64))), "plaquette_matrix")
    return out


def su3_path_holonomy(extents, links, start, steps):
    s = np.ascontiguousarray(steps, np.int32)
    out = np.zeros((3, 3), np.complex128)
    end = np.zeros(4, np.int64)
    _check(lib().or_su3_path_holonomy(_ext(extents), _dp(links.view(np.float64)), _x(start),
                                      s.ctypes.data_as(P(C.c_int32)), len(s),
                                      _dp(out.view(np.float64)),
                                      end.ctypes.data_as(P(i64))), "path_holonomy")
    return out, tuple(int(v) for v in end)


def rectangular_path(mu, nu, r, t) -> np.ndarray:
    steps = np.zeros(2 * (r + t) + 8, np.int32)
    n = i64()
    _check(lib().or_rectangular_path(mu, nu, r, t, steps.ctypes.data_as(P(C.c_int32)),
                                     len(steps), C.byref(n)), "rectangular_path")
    return steps[: n.value].copy()


def su3_wilson_loop(extents, links, start, steps) -> complex:
    s = np.ascontiguousarray(steps, np.int32)
    re, im = f64(), f64()
    _check(lib().or_su3_wilson_loop(_ext(extents), _dp(links.view(np.float64)), _x(start),
                                    s.ctypes.data_as(P(C.c_int32)), len(s), C.byref(re),
                                    C.byref(im)), "wilson_loop")
    return complex(re.value, im.value)


def su3_local_action_difference(extents, links, x, mu, candidate, beta) -> float:
    cand = np.ascontiguousarray(candidate, np.complex128)
    out = f64()
    _check(lib().or_su3_local_action_difference(_ext(extents), _dp(links.view(np.float64)),
                                                _x(x), mu, _dp(cand.view(np.float64)), beta,
                                                C.byref(out)), "local_action_difference")
    return out.value


def su3_metropolis_sweep(extents, links, beta, angle, rng_state: int):
    s, p, a = u64(rng_state), u64(), u64()
    _check(lib().or_su3_metropolis_sweep(_ext(extents), _dp(links.view(np.float64)), beta, angle,
                                         C.byref(s), C.byref(p), C.byref(a)), "metropolis_sweep")
    return s.value, p.value, a.value


def su3_run_chain(cfg: dict):
    c = Su3Config()
    c.extents = (i64 * 4)(*cfg["extents"])
    for k in ("beta", "master_seed", "chain_id", "thermalization_sweeps", "measurements",
              "sweeps_between_measurements", "proposal_angle", "autocorrelation_max_lag"):
        setattr(c, k, cfg[k])
    links = su3_links(n_links(cfg["extents"]))
    meas = np.zeros(cfg["measurements"], np.float64)
    out = Su3Scalars()
    _check(lib().or_su3_run_chain(C.byref(c), _dp(links.view(np.float64)), _dp(meas),
                                  C.byref(out)), "su3 run_chain")
    return links, meas, out


def su3_staple(extents, links, x, mu) -> np.ndarray:
    out = np.zeros((3, 3), np.complex128)
    _check(lib().or_su3_staple(_ext(extents), _dp(links.view(np.float64)), _x(x), mu,
                               _dp(out.view(np.float64))), "staple")
    return out


def su3_visit(u, a, beta, angle, key, uniform_generator=False):
    """One link visit of the checkerboard sweep (or_b200.c su3_visit): U after
    its eight hits given the staple sum A and the link's stream key, and the
    number of accepted hits."""
    uu = np.ascontiguousarray(u, np.complex128).copy()
    aa = np.ascontiguousarray(a, np.complex128)
    acc = u64()
    _check(lib().or_su3_visit(_dp(uu.view(np.float64)), _dp(aa.view(np.float64)), beta, angle,
                              key, int(uniform_generator), C.byref(acc)), "su3_visit")
    return uu, acc.value


def su3_cb_sweep(extents, links, beta, angle, chain_seed, sweep, uniform_generator=False):
    p, a = u64(), u64()
    _check(lib().or_su3_cb_sweep(_ext(extents), _dp(links.view(np.float64)), beta, angle,
                                 chain_seed, sweep, int(uniform_generator), C.byref(p),
                                 C.byref(a)), "cb_sweep")
    return p.value, a.value


# ---------------------------------------------------------------- SU(2)

def su2_identity(extents) -> np.ndarray:
    links = np.zeros((n_links(extents), 4), np.float64)
    links[:, 0] = 1.0
    return links


def su2_from_axis_angle(axis, angle) -> np.ndarray:
    a = np.ascontiguousarray(axis, np.float64)
    out = np.zeros(4, np.float64)
    _check(lib().or_su2_from_axis_angle(_dp(a), angle, _dp(out)), "from_axis_angle")
    return out


def su2_average_plaquette(extents, links) -> float:
    out = f64()
    _check(lib().or_su2_average_plaquette(_ext(extents), _dp(links), C.byref(out)),
           "su2 average_plaquette")
    return out.value


def su2_wilson_action(extents, links, beta) -> float:
    out = f64()
    _check(lib().or_su2_wilson_action(_ext(extents), _dp(links), beta, C.byref(out)),
           "su2 wilson_action")
    return out.value


def su2_wilson_loop(extents, links, start, steps) -> float:
    s = np.ascontiguousarray(steps, np.int32)
    out = f64()
    _check(lib().or_su2_wilson_loop(_ext(extents), _dp(links), _x(start),
                                    s.ctypes.data_as(P(C.c_int32)), len(s), C.byref(out)),
           "su2 wilson_loop")
    return out.value


def su2_polyakov_loop(extents, links, start, direction) -> float:
    out = f64()
    _check(lib().or_su2_polyakov_loop(_ext(extents), _dp(links), _x(start), direction,
                                      C.byref(out)), "su2 polyakov")
    return out.value


def su2_plaquette(extents, links, x, mu, nu) -> np.ndarray:
    out = np.zeros(4, np.float64)
    _check(lib().or_su2_plaquette(_ext(extents), _dp(links), _x(x), mu, nu, _dp(out)),
           "su2 plaquette")
    return out


def su2_staple(extents, links, x, mu) -> np.ndarray:
    out = np.zeros(4, np.float64)
    _check(lib().or_su2_staple(_ext(extents), _dp(links), _x(x), mu, _dp(out)), "su2 staple")
    return out


def su2_max_unit_residual(extents, links) -> float:
    out = f64()
    _check(lib().or_su2_max_unit_residual(_ext(extents), _dp(links), C.byref(out)), "residual")
    return out.value


def su2_heatbath_sweep(extents, links, beta, rng_state, max_attempts):
    s, p, u = u64(rng_state), u64(), u64()
    _check(lib().or_su2_heatbath_sweep(_ext(extents), _dp(links), beta, C.byref(s), max_attempts,
                                       C.byref(p), C.byref(u)), "heatbath_sweep")
    return s.value, p.value, u.value


def su2_overrelaxation_sweep(extents, links) -> None:
    _check(lib().or_su2_overrelaxation_sweep(_ext(extents), _dp(links)), "overrelaxation_sweep")


def su2_cb_sweep(extents, links, beta, chain_seed, sweep, overrelaxation_sweeps, max_attempts):
    p = u64()
    L = lib()
    L.or_su2_cb_sweep.argtypes = [P(i64), P(f64), f64, u64, u64, i64, i64, P(u64)]
    _check(L.or_su2_cb_sweep(_ext(extents), _dp(links), beta, chain_seed, sweep,
                             overrelaxation_sweeps, max_attempts, C.byref(p)), "su2 cb_sweep")
    return p.value


def su2_run_chain(cfg: dict):
    c = Su2Config()
    c.extents = (i64 * 4)(*cfg["extents"])
    for k in ("beta", "master_seed", "chain_id", "thermalization_sweeps", "measurements",
              "sweeps_between_measurements", "overrelaxation_sweeps_per_heatbath",
              "max_heatbath_attempts_per_link", "autocorrelation_max_lag"):
        setattr(c, k, cfg[k])
    links = np.zeros((n_links(cfg["extents"]), 4), np.float64)
    meas = np.zeros(cfg["measurements"], np.float64)
    out = Su2Scalars()
    _check(lib().or_su2_run_chain(C.byref(c), _dp(links), _dp(meas), C.byref(out)),
           "su2 run_chain")
    return links, meas, out


# ---------------------------------------------------------------- statistics

def diagnostics(values, max_lag):
    v = np.ascontiguousarray(values, np.float64)
    ac = np.zeros(max_lag + 1, np.float64)
    out = Diagnostics()
    _check(lib().or_diagnostics(_dp(v), len(v), max_lag, C.byref(out), _dp(ac)), "diagnostics")
    return out, ac


def sampling_efficiency(values, log_weights, max_lag, setup, thermalization, sampling):
    v = np.ascontiguousarray(values, np.float64)
    w = None if log_weights is None else np.ascontiguousarray(log_weights, np.float64)
    ac = np.zeros(max_lag + 1, np.float64)
    out = Efficiency()
    _check(lib().or_sampling_efficiency(_dp(v), len(v), None if w is None else _dp(w), max_lag,
                                        setup, thermalization, sampling, C.byref(out), _dp(ac)),
           "sampling_efficiency")
    return out


def periodic_connected_estimator(samples: np.ndarray):
    s = np.ascontiguousarray(samples, np.float64)
    ncfg, nt = s.shape
    vac = f64()
    raw = np.zeros(nt)
    con = np.zeros(nt)
    _check(lib().or_periodic_connected_estimator(_dp(s), ncfg, nt, C.byref(vac), _dp(raw),
                                                 _dp(con)), "periodic estimator")
    return vac.value, raw, con


def connected_from_samples(samples: np.ndarray, omitted=None) -> np.ndarray:
    s = np.ascontiguousarray(samples, np.float64)
    ncfg, nt = s.shape
    con = np.zeros(nt)
    _check(lib().or_connected_from_samples(_dp(s), ncfg, nt, -1 if omitted is None else omitted,
                                           _dp(con)), "connected_from_samples")
    return con


def jackknife_covariance(replicas: np.ndarray, start: int, end: int) -> np.ndarray:
    r = np.ascontiguousarray(replicas, np.float64)
    nrep, nt = r.shape
    pts = end - start + 1
    out = np.zeros((pts, pts))
    _check(lib().or_jackknife_covariance(_dp(r), nrep, nt, start, end, _dp(out)),
           "jackknife_covariance")
    return out


# ---------------------------------------------------------------- glueball

def scalar_a1pp_operator_basis(extents, links, t):
    p, r = f64(), f64()
    pc, rc = i64(), i64()
    _check(lib().or_scalar_a1pp_operator_basis(_ext(extents), _dp(links.view(np.float64)), t,
                                               C.byref(p), C.byref(r), C.byref(pc), C.byref(rc)),
           "operator_basis")
    return p.value, r.value, pc.value, rc.value


def spatial_stout_smear(extents, links, rho, levels, lift_level_cap=False) -> np.ndarray:
    out = np.empty_like(links)
    _check(lib().or_spatial_stout_smear(_ext(extents), _dp(links.view(np.float64)), rho, levels,
                                        int(lift_level_cap), _dp(out.view(np.float64))),
           "stout_smear")
    return out


def max_link_residual(extents, a, b) -> float:
    out = f64()
    _check(lib().or_max_link_residual(_ext(extents), _dp(a.view(np.float64)),
                                      _dp(b.view(np.float64)), C.byref(out)), "max_link_residual")
    return out.value


def spatial_stride2_block(extents, links):
    cext = (i64 * 4)()
    _check(lib().or_blocked_extents(_ext(extents), cext), "blocked_extents")
    coarse_ext = [cext[i] for i in range(4)]
    out = su3_links(n_links(coarse_ext))
    _check(lib().or_spatial_stride2_block(_ext(extents), _dp(links.view(np.float64)),
                                          _dp(out.view(np.float64))), "stride2_block")
    return coarse_ext, out


def scalar_connected_correlators(extents, configs):
    cfgs = np.ascontiguousarray(np.stack(configs), np.complex128)
    nt = extents[3]
    vac = np.zeros(2)
    raw = np.zeros(2 * nt)
    con = np.zeros(2 * nt)
    _check(lib().or_scalar_connected_correlators(_ext(extents), _dp(cfgs.view(np.float64)),
                                                 len(configs), _dp(vac), _dp(raw), _dp(con)),
           "scalar_connected_correlators")
    return vac, raw.reshape(2, nt), con.reshape(2, nt)


def bench_su3_reference(extents, beta, angle, master_seed, threads, links_per_thread):
    secs, done = f64(), u64()
    _check(lib().or_bench_su3_reference(_ext(extents), beta, angle, master_seed, threads,
                                        links_per_thread, C.byref(secs), C.byref(done)),
           "bench_su3_reference")
    return secs.value, done.value


# ---------------------------------------------------------------- learned proposal

LP_PARAMS = 6288
LP_OFF = {"W1": 0, "b1": 1024, "W2": 1088, "b2": 5184, "W3": 5248, "b3": 6272}


def _f32(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"] and a.dtype == np.float32
    return a.ctypes.data_as(P(C.c_float))


def bf16_round(x) -> np.ndarray:
    """binary32 -> bfloat16 -> binary32, round to nearest even (vectorised)."""
    a = np.ascontiguousarray(x, np.float32).copy()
    b = a.view(np.uint32)
    finite = (b & 0x7F800000) != 0x7F800000
    r = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    b[finite] = r[finite]
    return a


def lp_features(staple18, beta) -> np.ndarray:
    a = np.ascontiguousarray(staple18, np.complex128)
    f = np.zeros(16)
    _check(lib().or_lp_features(_dp(a.view(np.float64)), f64(beta), _dp(f)), "lp_features")
    return f


def lp_forward(params, features) -> np.ndarray:
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(features, np.float32).reshape(-1, 16)
    y = np.zeros((x.shape[0], 16))
    L = lib()
    L.or_lp_forward.argtypes = [P(C.c_float), P(C.c_float), i64, P(f64)]
    _check(L.or_lp_forward(_f32(p), _f32(x), x.shape[0], _dp(y)), "lp_forward")
    return y


def lp_proposal(y16):
    y = np.ascontiguousarray(y16, np.float64)
    p = np.zeros(8)
    s = f64()
    _check(lib().or_lp_proposal(_dp(y), _dp(p), C.byref(s)), "lp_proposal")
    return p, s.value


def lp_retr_rotated(g, m18, theta):
    m = np.ascontiguousarray(m18, np.float32).reshape(18)
    f, df = f64(), f64()
    L = lib()
    L.or_lp_retr_rotated.argtypes = [C.c_int, P(C.c_float), f64, P(f64), P(f64)]
    _check(L.or_lp_retr_rotated(g, _f32(m), theta, C.byref(f), C.byref(df)), "lp_retr_rotated")
    return f.value, df.value


def lp_loss_grad(params, features, m18, beta, exact=False):
    """Objective and gradient with the device's BF16 roundings (exact=False)
    or in plain binary64 arithmetic on binary32 inputs (exact=True)."""
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(features, np.float32).reshape(-1, 16)
    m = np.ascontiguousarray(m18, np.float32).reshape(-1, 18)
    b = np.ascontiguousarray(np.broadcast_to(np.asarray(beta, np.float64), (x.shape[0],)))
    g = np.zeros(LP_PARAMS)
    obj = f64()
    L = lib()
    L.or_lp_loss_grad_mode.argtypes = [P(C.c_float), P(C.c_float), P(C.c_float), P(f64), i64,
                                       C.c_int, P(f64), P(f64)]
    _check(L.or_lp_loss_grad_mode(_f32(p), _f32(x), _f32(m), _dp(b), x.shape[0], int(exact),
                                  C.byref(obj), _dp(g)), "lp_loss_grad")
    return obj.value, g


def lp_objective_exact(params, features, m18, beta) -> float:
    p = np.ascontiguousarray(params, np.float64)
    x = np.ascontiguousarray(features, np.float64).reshape(-1, 16)
    m = np.ascontiguousarray(m18, np.float32).reshape(-1, 18)
    b = np.ascontiguousarray(np.broadcast_to(np.asarray(beta, np.float64), (x.shape[0],)))
    obj = f64()
    L = lib()
    L.or_lp_objective_exact.argtypes = [P(f64), P(f64), P(C.c_float), P(f64), i64, P(f64)]
    _check(L.or_lp_objective_exact(_dp(p), _dp(x), _f32(m), _dp(b), x.shape[0], C.byref(obj)),
           "lp_objective_exact")
    return obj.value


def lp_pick_generator(word, p8) -> int:
    p = np.ascontiguousarray(p8, np.float64)
    L = lib()
    L.or_lp_pick_generator.argtypes = [u64, P(f64)]
    return int(L.or_lp_pick_generator(word, _dp(p)))


def lp_cb_sweep(extents, links, beta, params, chain_seed, sweep):
    p = np.ascontiguousarray(params, np.float32)
    npr, nac = u64(), u64()
    L = lib()
    L.or_lp_cb_sweep.argtypes = [P(i64), P(f64), f64, P(C.c_float), u64, u64, P(u64), P(u64)]
    _check(L.or_lp_cb_sweep(_ext(extents), _dp(links.view(np.float64)), beta, _f32(p), chain_seed,
                            sweep, C.byref(npr), C.byref(nac)), "lp_cb_sweep")
    return npr.value, nac.value


def su3_hit(u18, staple18, beta, angle, w_angle, w_acc, g):
    u = np.ascontiguousarray(u18, np.complex128).copy()
    a = np.ascontiguousarray(staple18, np.complex128)
    acc = u64()
    L = lib()
    L.or_su3_hit.argtypes = [P(f64), P(f64), f64, f64, u64, u64, C.c_int, P(u64)]
    _check(L.or_su3_hit(_dp(u.view(np.float64)), _dp(a.view(np.float64)), beta, angle, w_angle,
                        w_acc, g, C.byref(acc)), "su3_hit")
    return u, bool(acc.value)
