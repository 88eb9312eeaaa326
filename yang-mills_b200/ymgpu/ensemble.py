"""Device ensembles: one or more lattices (chains) held on a B200.

``Ensemble`` wraps the opaque ``ym_ensemble`` handle of libymgpu.  A chain is
one reference lattice (``Su3Lattice4`` / ``Lattice4``); many chains of uneven
extents share one handle and are updated by the same kernel launches.  Host
lattices cross the boundary as numpy arrays in the reference's memory order:
SU(3) ``(links, 3, 3)`` complex128, link index ``site*4 + mu`` with
lexicographic sites, x3 fastest.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from ._lib import EnsembleDesc, GlueballPlan, MeasuredRun, lib
from .errors import check

SU2, SU3 = 2, 3
F64, F32_TWO_ROW = 0, 1
ORDERED, UNIFORM = 0, 1
_GEN = {"ordered": ORDERED, "uniform": UNIFORM, ORDERED: ORDERED, UNIFORM: UNIFORM}


def _f64p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _u64p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _i64p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _site(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.int64).reshape(4))


def _steps(steps) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(steps, dtype=np.int32).reshape(-1))


class Ensemble:
    """A set of chains resident in device memory (see include/ymgpu.h)."""

    def __init__(self, extents: Sequence[Sequence[int]], beta, seeds, group: int = SU3,
                 precision: int = F64, lift_reference_caps: bool = False, device: int = 0):
        ext = np.ascontiguousarray(np.asarray(extents, dtype=np.int64).reshape(-1, 4))
        n = ext.shape[0]
        betas = np.ascontiguousarray(np.broadcast_to(np.asarray(beta, np.float64), (n,)).copy())
        sd = np.ascontiguousarray(np.broadcast_to(np.asarray(seeds, np.uint64), (n,)).copy())
        desc = EnsembleDesc(group, precision, n, ext.ctypes.data_as(C.POINTER(C.c_int64)),
                            _f64p(betas), _u64p(sd), int(lift_reference_caps), device)
        h = C.c_void_p()
        check(lib().ym_ensemble_create(C.byref(desc), C.byref(h)), "ym_ensemble_create")
        self._h = h
        self.extents = [tuple(int(v) for v in row) for row in ext]
        self.beta = betas
        self.seeds = sd
        self.group = group
        self.precision = precision
        self.n_chains = n
        self.device = device

    # ------------------------------------------------------------ lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib().ym_ensemble_destroy(self._h), "ym_ensemble_destroy")
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def links_in_chain(self, chain: int) -> int:
        return int(np.prod(self.extents[chain])) * 4

    # ------------------------------------------------------------ state
    def set_identity(self) -> None:
        check(lib().ym_ensemble_set_identity(self._h), "set_identity")

    def hot_start(self) -> None:
        check(lib().ym_ensemble_hot_start(self._h), "hot_start")

    def upload(self, chain: int, links: np.ndarray) -> None:
        """SU(3): (links, 3, 3) complex128; SU(2): (links, 4) float64 quaternions."""
        if self.group == SU3:
            a = np.ascontiguousarray(links, dtype=np.complex128)
            ok = a.size == self.links_in_chain(chain) * 9
            a = a.view(np.float64)
        else:
            a = np.ascontiguousarray(links, dtype=np.float64)
            ok = a.size == self.links_in_chain(chain) * 4
        if not ok:
            raise ValueError("link array does not match the chain's extents")
        check(lib().ym_ensemble_upload(self._h, chain, _f64p(a)), "upload")

    def download(self, chain: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = (np.empty((self.links_in_chain(chain), 3, 3), np.complex128) if self.group == SU3
                   else np.empty((self.links_in_chain(chain), 4), np.float64))
        buf = out.view(np.float64) if out.dtype == np.complex128 else out
        check(lib().ym_ensemble_download(self._h, chain, _f64p(buf)), "download")
        return out

    def set_chain(self, chain: int, beta: float, seed: int) -> None:
        check(lib().ym_ensemble_set_chain(self._h, chain, float(beta), int(seed)), "set_chain")
        self.beta[chain] = beta
        self.seeds[chain] = seed

    @property
    def sweep_index(self) -> int:
        v = C.c_uint64()
        check(lib().ym_ensemble_get_sweep_index(self._h, C.byref(v)), "get_sweep_index")
        return v.value

    @sweep_index.setter
    def sweep_index(self, value: int) -> None:
        check(lib().ym_ensemble_set_sweep_index(self._h, int(value)), "set_sweep_index")

    def synchronize(self) -> None:
        check(lib().ym_ensemble_synchronize(self._h), "synchronize")

    def stream(self) -> int:
        p = C.c_void_p()
        check(lib().ym_ensemble_stream(self._h, C.byref(p)), "stream")
        return p.value or 0

    # ------------------------------------------------------------ SU(3) updates
    def metropolis_sweeps(self, proposal_angle: float, n_sweeps: int = 1,
                          generator_mode="ordered") -> None:
        check(lib().ym_su3_metropolis_sweeps(self._h, float(proposal_angle), _GEN[generator_mode],
                                             int(n_sweeps)), "su3_metropolis_sweeps")

    def measured_sweeps(self, proposal_angle: float, n_measurements: int,
                        sweeps_per_measurement: int = 1, generator_mode="ordered") -> np.ndarray:
        """[measurement, chain] plaquette series of a graph-replayed cadence."""
        out = np.zeros((n_measurements, self.n_chains), np.float64)
        check(lib().ym_su3_measured_sweeps(self._h, float(proposal_angle), _GEN[generator_mode],
                                           int(n_measurements), int(sweeps_per_measurement),
                                           _f64p(out)), "su3_measured_sweeps")
        return out

    def measured_run(self, proposal_angle: float, n_blocks: int, sweeps_per_block: int = 10,
                     rmax: int = 4, tmax: int = 4, polyakov_direction: int = 3,
                     generator_mode="ordered", view: "Ensemble" = None):
        """Sweeps with the plaquette after each, and Wilson (R x T <= rmax x tmax)
        and Polyakov loops after every block of sweeps, one captured graph per
        block (include/ymgpu.h ym_su3_measured_run).  A two-row handle needs
        a binary64 ``view`` of the same extents for the loops.  Returns
        (plaquette [sweep, chain], wilson [block, chain, plane, R-1, T-1],
        polyakov [block, chain] complex)."""
        run = MeasuredRun(float(proposal_angle), _GEN[generator_mode], int(polyakov_direction),
                          int(n_blocks), int(sweeps_per_block), int(rmax), int(tmax))
        plaq = np.zeros((n_blocks * sweeps_per_block, self.n_chains), np.float64)
        wil = np.zeros((n_blocks, self.n_chains, 6, 4, 4), np.float64)
        pol = np.zeros((n_blocks, self.n_chains, 2), np.float64)
        check(lib().ym_su3_measured_run(self._h, view.handle if view is not None else None,
                                        C.byref(run), _f64p(plaq), _f64p(wil), _f64p(pol)),
              "su3_measured_run")
        return plaq, wil, pol[..., 0] + 1j * pol[..., 1]

    @property
    def sweep_layout(self) -> dict:
        """The SU(3) FP64 sub-sweep's work layout: item size, order, tuned."""
        n, v, t = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().ym_ensemble_get_sweep_layout(self._h, C.byref(n), C.byref(v), C.byref(t)),
              "get_sweep_layout")
        return {"item_sites": n.value, "by_volume": bool(v.value), "tuned": bool(t.value)}

    def set_sweep_layout(self, item_sites: int = 0, by_volume: bool = False) -> None:
        """Force a layout (item_sites 128/64/32) or ask for tuning (0)."""
        check(lib().ym_ensemble_set_sweep_layout(self._h, int(item_sites), int(by_volume)),
              "set_sweep_layout")

    def lift_angle_cap(self, lift: bool = True) -> None:
        """Admit half widths up to 2.5 on a two-row handle (past the
        reference's 1.0), for plain Metropolis at a learned scale."""
        check(lib().ym_ensemble_lift_angle_cap(self._h, int(lift)), "lift_angle_cap")

    @property
    def fast_sweeps(self) -> bool:
        """Whether SU(3) FP64 sweeps run in the fast form (fused
        multiply-adds, Horner rotations; a few ulps per update from the
        reference's bits, include/ymgpu.h) instead of the exact one."""
        v = C.c_int32()
        check(lib().ym_ensemble_get_fast_sweeps(self._h, C.byref(v)), "get_fast_sweeps")
        return bool(v.value)

    @fast_sweeps.setter
    def fast_sweeps(self, on: bool) -> None:
        check(lib().ym_ensemble_set_fast_sweeps(self._h, int(bool(on))), "set_fast_sweeps")

    @property
    def sweep_path(self) -> str:
        """'auto' (undecided), 'tiled' or 'resident' (include/ymgpu.h)."""
        v = C.c_int32()
        check(lib().ym_ensemble_get_sweep_path(self._h, C.byref(v)), "get_sweep_path")
        return {-1: "auto", 0: "tiled", 1: "resident"}[v.value]

    @sweep_path.setter
    def sweep_path(self, value: str) -> None:
        check(lib().ym_ensemble_set_sweep_path(self._h, {"auto": -1, "tiled": 0, "resident": 1}[value]),
              "set_sweep_path")

    def accounting(self):
        p = np.zeros(self.n_chains, np.uint64)
        a = np.zeros(self.n_chains, np.uint64)
        check(lib().ym_su3_accounting(self._h, _u64p(p), _u64p(a)), "su3_accounting")
        return p, a

    def reset_accounting(self) -> None:
        check(lib().ym_reset_accounting(self._h), "reset_accounting")

    def reference_sweeps(self, proposal_angle: float, rng_state, n_sweeps: int = 1):
        st = np.ascontiguousarray(np.broadcast_to(np.asarray(rng_state, np.uint64),
                                                  (self.n_chains,)).copy())
        p = np.zeros(self.n_chains, np.uint64)
        a = np.zeros(self.n_chains, np.uint64)
        check(lib().ym_su3_reference_sweeps(self._h, float(proposal_angle), _u64p(st),
                                            int(n_sweeps), _u64p(p), _u64p(a)),
              "su3_reference_sweeps")
        return st, p, a

    # ------------------------------------------------------------ SU(2) updates
    def markov_sweeps(self, n_sweeps: int = 1, overrelaxation_sweeps: int = 1,
                      max_attempts_per_link: int = 10000, sampler: str = "reference") -> None:
        """Heat-bath + overrelaxation sweeps (su2_ensemble.rs:465-486)."""
        code = {"reference": 0, "kennedy-pendleton": 1}[sampler]
        check(lib().ym_su2_markov_sweeps(self._h, int(max_attempts_per_link),
                                         int(overrelaxation_sweeps), code, int(n_sweeps)),
              "su2_markov_sweeps")

    def su2_measured_sweeps(self, n_measurements: int, sweeps_per_measurement: int = 1,
                            overrelaxation_sweeps: int = 1, max_attempts_per_link: int = 10000,
                            sampler: str = "reference") -> np.ndarray:
        """run_chain's cadence on the device: n_measurements times
        {sweeps_per_measurement markov_sweeps, average plaquette}, one
        captured graph; returns the series [measurement, chain]."""
        code = {"reference": 0, "kennedy-pendleton": 1}[sampler]
        out = np.zeros((int(n_measurements), self.n_chains), np.float64)
        check(lib().ym_su2_measured_sweeps(self._h, int(max_attempts_per_link), int(overrelaxation_sweeps), code,
                                           int(n_measurements), int(sweeps_per_measurement), _f64p(out)),
              "su2_measured_sweeps")
        return out

    def overrelaxation_sweeps(self, n_sweeps: int = 1) -> None:
        check(lib().ym_su2_overrelaxation_sweeps(self._h, int(n_sweeps)), "su2_overrelaxation")

    def heatbath_accounting(self):
        p = np.zeros(self.n_chains, np.uint64)
        u = np.zeros(self.n_chains, np.uint64)
        check(lib().ym_su2_accounting(self._h, _u64p(p), _u64p(u)), "su2_accounting")
        return p, u

    def max_unit_residual(self) -> np.ndarray:
        out = np.zeros(self.n_chains, np.float64)
        check(lib().ym_su2_max_unit_residual(self._h, _f64p(out)), "su2_max_unit_residual")
        return out

    # ------------------------------------------------------------ timing
    def profile(self, on: bool = True) -> None:
        check(lib().ym_profile_enable(self._h, int(on)), "profile_enable")

    def profile_read(self, kernel: str):
        """(total device ms, launches) of one kernel since the last read."""
        from ._lib import KERNEL_IDS
        ms, n = C.c_double(), C.c_int64()
        check(lib().ym_profile_read(self._h, KERNEL_IDS[kernel], C.byref(ms), C.byref(n)),
              "profile_read")
        return ms.value, n.value

    # ------------------------------------------------------------ observables
    def average_plaquette(self) -> np.ndarray:
        out = np.zeros(self.n_chains, np.float64)
        check(lib().ym_average_plaquette(self._h, _f64p(out)), "average_plaquette")
        return out

    def wilson_loops(self, rmax: int = 4, tmax: int = 4) -> np.ndarray:
        """[chain, plane, R-1, T-1] lattice means of Re W(R x T); planes
        (0,1),(0,2),(0,3),(1,2),(1,3),(2,3), R along the first direction."""
        out = np.zeros(self.n_chains * 96, np.float64)
        check(lib().ym_su3_wilson_loops(self._h, rmax, tmax, _f64p(out)), "wilson_loops")
        return out.reshape(self.n_chains, 6, 4, 4)

    def polyakov_loops(self, direction: int = 3) -> np.ndarray:
        out = np.zeros(self.n_chains * 2, np.float64)
        check(lib().ym_su3_polyakov_loops(self._h, direction, _f64p(out)), "polyakov_loops")
        return out[0::2] + 1j * out[1::2]

    def scalar_operator_basis(self):
        """Per chain: (plaquette[t], rectangle[t]) time-slice means."""
        n = sum(e[3] for e in self.extents)
        p = np.zeros(n, np.float64)
        r = np.zeros(n, np.float64)
        check(lib().ym_su3_scalar_operator_basis(self._h, _f64p(p), _f64p(r)), "operator_basis")
        out, k = [], 0
        for e in self.extents:
            out.append((p[k:k + e[3]].copy(), r[k:k + e[3]].copy()))
            k += e[3]
        return out

    # ------------------------------------------------------------ per-site / per-link queries
    def _link_reals(self) -> int:
        return 18 if self.group == SU3 else 4

    def _as_link(self, a: np.ndarray):
        """Host form of one link: (3, 3) complex128 (SU(3)) or 4 float64."""
        return a.view(np.complex128).reshape(3, 3) if self.group == SU3 else a

    def get_link(self, chain: int, x, mu: int) -> np.ndarray:
        """One link, moved alone (Su3Lattice4::link su3_lattice.rs:153-155)."""
        out = np.zeros(self._link_reals(), np.float64)
        check(lib().ym_ensemble_get_link(self._h, chain, _i64p(_site(x)), mu, _f64p(out)), "get_link")
        return self._as_link(out)

    def set_link(self, chain: int, x, mu: int, value) -> None:
        """Su3Lattice4::set_link (su3_lattice.rs:157-166): one link, moved alone."""
        dt = np.complex128 if self.group == SU3 else np.float64
        v = np.ascontiguousarray(np.asarray(value, dtype=dt)).reshape(-1).view(np.float64)
        if v.size != self._link_reals():
            raise ValueError("link value has the wrong size for the group")
        check(lib().ym_ensemble_set_link(self._h, chain, _i64p(_site(x)), mu, _f64p(v)), "set_link")

    def path_holonomy(self, chain: int, start, steps):
        """(holonomy, end) of path_holonomy (path_holonomy.rs:132-161)."""
        st = _steps(steps)
        hol = np.zeros(self._link_reals(), np.float64)
        end = np.zeros(4, np.int64)
        check(lib().ym_path_holonomy(self._h, chain, _i64p(_site(start)),
                                     st.ctypes.data_as(C.POINTER(C.c_int32)), st.size, _f64p(hol),
                                     _i64p(end)), "path_holonomy")
        return self._as_link(hol), tuple(int(v) for v in end)

    def wilson_loop(self, chain: int, start, steps) -> complex:
        """wilson_loop (path_holonomy.rs:172-181): (1/3) Tr (SU(3)) or (1/2) Re Tr (SU(2))."""
        st = _steps(steps)
        out = np.zeros(2, np.float64)
        check(lib().ym_wilson_loop(self._h, chain, _i64p(_site(start)),
                                   st.ctypes.data_as(C.POINTER(C.c_int32)), st.size, _f64p(out)),
              "wilson_loop")
        return complex(out[0], out[1])

    def wilson_loop_sites(self, chain: int, steps) -> np.ndarray:
        """wilson_loop from every site of the chain, lexicographic order (complex128)."""
        st = _steps(steps)
        out = np.zeros(2 * int(np.prod(self.extents[chain])), np.float64)
        check(lib().ym_wilson_loop_sites(self._h, chain, st.ctypes.data_as(C.POINTER(C.c_int32)),
                                         st.size, _f64p(out)), "wilson_loop_sites")
        return out.view(np.complex128)

    def polyakov_loop(self, chain: int, start, direction: int) -> complex:
        """Su3Lattice4::polyakov_loop (su3_lattice.rs:202-212) / Lattice4::polyakov_loop."""
        out = np.zeros(2, np.float64)
        check(lib().ym_polyakov_loop(self._h, chain, _i64p(_site(start)), direction, _f64p(out)),
              "polyakov_loop")
        return complex(out[0], out[1])

    def polyakov_loop_sites(self, chain: int, direction: int) -> np.ndarray:
        out = np.zeros(2 * int(np.prod(self.extents[chain])), np.float64)
        check(lib().ym_polyakov_loop_sites(self._h, chain, direction, _f64p(out)),
              "polyakov_loop_sites")
        return out.view(np.complex128)

    def plaquette_at(self, chain: int, x, mu: int, nu: int) -> np.ndarray:
        """plaquette(x, mu, nu): SU(3) matrix / SU(2) quaternion."""
        out = np.zeros(self._link_reals(), np.float64)
        check(lib().ym_plaquette(self._h, chain, _i64p(_site(x)), mu, nu, _f64p(out)), "plaquette")
        return self._as_link(out)

    def wilson_action(self, beta: float) -> np.ndarray:
        """wilson_action(beta) of every chain, the reference's sequential sum."""
        out = np.zeros(self.n_chains, np.float64)
        check(lib().ym_wilson_action(self._h, float(beta), _f64p(out)), "wilson_action")
        return out

    def su2_staple(self, chain: int, x, mu: int):
        """Lattice4::staple (lib.rs:507-546): (components, terms)."""
        out = np.zeros(4, np.float64)
        terms = C.c_int64()
        check(lib().ym_su2_staple(self._h, chain, _i64p(_site(x)), mu, _f64p(out), C.byref(terms)),
              "su2_staple")
        return out, terms.value

    def local_link_action(self, chain: int, x, mu: int, beta: float) -> float:
        out = np.zeros(1, np.float64)
        check(lib().ym_su3_local_link_action(self._h, chain, _i64p(_site(x)), mu, float(beta),
                                             _f64p(out)), "local_link_action")
        return float(out[0])

    def local_action_difference(self, chain: int, x, mu: int, candidate, beta: float) -> float:
        """local_action_difference (su3_ensemble.rs:319-334)."""
        cand = np.ascontiguousarray(np.asarray(candidate, dtype=np.complex128)).reshape(-1).view(np.float64)
        out = np.zeros(1, np.float64)
        check(lib().ym_su3_local_action_difference(self._h, chain, _i64p(_site(x)), mu, _f64p(cand),
                                                   float(beta), _f64p(out)),
              "local_action_difference")
        return float(out[0])

    def gauge_transform(self, chain: int, site_gauges, dst: "Ensemble" = None,
                        dst_chain: int = None) -> None:
        """Su3Lattice4::gauge_transform (su3_lattice.rs:244-283) into dst (default: in place);
        site_gauges is (V, 3, 3) complex128 in lexicographic site order."""
        g = np.ascontiguousarray(np.asarray(site_gauges, dtype=np.complex128)).view(np.float64)
        if g.size != int(np.prod(self.extents[chain])) * 18:
            raise ValueError("one SU(3) gauge per site is needed")
        dst = self if dst is None else dst
        dst_chain = chain if dst_chain is None else dst_chain
        check(lib().ym_su3_gauge_transform(self._h, chain, _f64p(g), dst.handle, dst_chain),
              "gauge_transform")

    def su2_wilson_loops(self, rmax: int = 4, tmax: int = 4) -> np.ndarray:
        """[chain, plane, R-1, T-1] lattice means of Lattice4::rectangular_wilson_loop."""
        out = np.zeros(self.n_chains * 96, np.float64)
        check(lib().ym_su2_wilson_loops(self._h, rmax, tmax, _f64p(out)), "su2_wilson_loops")
        return out.reshape(self.n_chains, 6, 4, 4)

    def su2_polyakov_loops(self, direction: int = 3) -> np.ndarray:
        out = np.zeros(self.n_chains, np.float64)
        check(lib().ym_su2_polyakov_loops(self._h, direction, _f64p(out)), "su2_polyakov_loops")
        return out

    def reunitarize(self) -> None:
        """Binary64 Gram-Schmidt of two-row binary32 links (YM_PREC_F32_TWO_ROW)."""
        check(lib().ym_su3_reunitarize(self._h), "reunitarize")

    def convert_to(self, dst: "Ensemble") -> None:
        """Copy into a handle of the same extents, converting precision."""
        check(lib().ym_ensemble_convert(self._h, dst.handle), "ensemble_convert")

    def copy_chain_to(self, chain: int, dst: "Ensemble", dst_chain: int) -> None:
        check(lib().ym_ensemble_copy_chain(self._h, chain, dst.handle, dst_chain), "copy_chain")

    def copy_chains_to(self, first: int, dst: "Ensemble", dst_first: int, count: int) -> None:
        """Copy chains first..first+count-1 into dst_first.. of dst (one copy)."""
        check(lib().ym_ensemble_copy_chains(self._h, first, dst.handle, dst_first, count),
              "copy_chains")

    def copy_subset_to(self, chains, dst: "Ensemble") -> None:
        """Copy the given chains into chains 0.. of dst, one copy per run of
        consecutive chain indices."""
        chains = list(chains)
        j = 0
        while j < len(chains):
            k = j
            while k + 1 < len(chains) and chains[k + 1] == chains[k] + 1:
                k += 1
            self.copy_chains_to(chains[j], dst, j, k - j + 1)
            j = k + 1

    def subset(self, chains) -> "Ensemble":
        """A new handle holding a device copy of the given chains."""
        chains = list(chains)
        out = Ensemble([self.extents[c] for c in chains], self.beta[chains], self.seeds[chains],
                       group=self.group, precision=self.precision, lift_reference_caps=True,
                       device=self.device)
        self.copy_subset_to(chains, out)
        return out

    def copy_to(self, dst: "Ensemble") -> None:
        check(lib().ym_ensemble_copy(self._h, dst.handle), "ensemble_copy")

    def stout_smear_into(self, dst: "Ensemble", rho: float, levels: int,
                         lift_level_cap: bool = False) -> None:
        check(lib().ym_su3_spatial_stout_smear(self._h, dst.handle, float(rho), int(levels),
                                               int(lift_level_cap)), "spatial_stout_smear")

    @staticmethod
    def _glueball_plan(levels, rho, blocked):
        lv = np.ascontiguousarray(np.asarray(levels, dtype=np.int64))
        blocked = list(blocked)
        fine = (C.c_void_p * max(1, len(blocked)))(*[b[0].handle.value for b in blocked])
        coarse = (C.c_void_p * max(1, len(blocked)))(*[b[1].handle.value for b in blocked])
        first = np.ascontiguousarray(np.asarray([b[2] for b in blocked] or [0], dtype=np.int64))
        plan = GlueballPlan(float(rho), len(lv), _i64p(lv), len(blocked), fine, coarse, _i64p(first))
        return plan, (lv, fine, coarse, first)       # the arrays the plan points into

    def glueball_prepare(self, smeared: "Ensemble", levels, rho: float = 0.1, blocked=()) -> None:
        """Build and upload the measurement graph of glueball_measure with
        these arguments without measuring (ym_su3_glueball_prepare)."""
        plan, keep = self._glueball_plan(levels, rho, blocked)
        check(lib().ym_su3_glueball_prepare(self._h, smeared.handle, C.byref(plan)), "glueball_prepare")
        del keep

    def glueball_measure(self, smeared: "Ensemble", levels, rho: float = 0.1, blocked=()):
        """One glueball measurement as one captured graph (ym_su3_glueball_measure):
        this handle's links smeared in place in `smeared` through the
        ascending level counts, the A1++ operator basis after each count, and
        for each (fine, coarse, first_chain) in `blocked` the chains
        first_chain.. of `smeared` blocked into `coarse` and measured.
        Returns (plaquette, rectangle, blocked_plaquette, blocked_rectangle),
        each [level, slice]."""
        blocked = list(blocked)
        plan, (lv, fine, coarse, first) = self._glueball_plan(levels, rho, blocked)
        n_sl = sum(e[3] for e in smeared.extents)
        n_bl = sum(sum(e[3] for e in b[1].extents) for b in blocked)
        p = np.zeros((len(lv), n_sl), np.float64)
        r = np.zeros((len(lv), n_sl), np.float64)
        bp = np.zeros((len(lv), max(n_bl, 1)), np.float64)
        br = np.zeros((len(lv), max(n_bl, 1)), np.float64)
        check(lib().ym_su3_glueball_measure(self._h, smeared.handle, C.byref(plan), _f64p(p), _f64p(r),
                                            _f64p(bp), _f64p(br)), "glueball_measure")
        return p, r, bp[:, :n_bl], br[:, :n_bl]

    def block_into(self, dst: "Ensemble") -> None:
        check(lib().ym_su3_spatial_stride2_block(self._h, dst.handle), "spatial_stride2_block")

    def like(self, extents=None, precision=None) -> "Ensemble":
        """A new handle with this one's chains (optionally other extents or
        storage precision)."""
        return Ensemble(extents if extents is not None else self.extents, self.beta, self.seeds,
                        group=self.group,
                        precision=self.precision if precision is None else precision,
                        lift_reference_caps=True, device=self.device)

    def reference_average_plaquette(self) -> np.ndarray:
        out = np.zeros(self.n_chains, np.float64)
        check(lib().ym_su3_reference_average_plaquette(self._h, _f64p(out)),
              "reference_average_plaquette")
        return out

    def max_residuals(self):
        u = np.zeros(self.n_chains, np.float64)
        d = np.zeros(self.n_chains, np.float64)
        check(lib().ym_su3_max_residuals(self._h, _f64p(u), _f64p(d)), "su3_max_residuals")
        return u, d
