"""Host-side mirror of the reference's per-step subroutine interface.

``System`` owns one device context (``mfa_ctx``) and exposes the subroutines
md_main.f90 calls, under the same names and in the same roles:

    verlet_positions, check_skin, binning, my_binning, fluid_fluid,
    fluid_wall(inter_type), intra_molec, bending(mode), ewald_k(mode),
    verlet_velocities

plus ``md_step`` (one iteration of md_main.f90:68-147 through those calls),
``step(n)`` (the fused, graph-captured device loop) and the host mirrors.
Every call goes through the C ABI of libmfa_gpu.so; errors raise MfaError,
the way the reference stops.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from ._abi import MfaParams, MfaScalars, check, load


def _dp(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int32))


class System:
    """One simulated system resident on one GPU."""

    def __init__(self, params: MfaParams, r0, v, a_type, mass, q=None, a=None, mic=None,
                 precision: int = _abi.MIXED, device: int = 0, bin_type: int = 0):
        if bin_type not in (0, 1):
            raise ValueError("bin_type is 0 (binning) or 1 (my_binning)")
        self.lib = load()
        # BIN_TYPE of control_simulation.h: the list rule of every rebuild this
        # object starts (init_forces, md_step, restore); calling binning() or
        # my_binning() directly switches it, as the library's context does
        self.bin_type = bin_type
        self.params = params.copy()
        self.n = int(params.n_part)
        self.precision = precision
        r0 = np.ascontiguousarray(r0, dtype=np.float64).reshape(self.n, 3)
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(self.n, 3)
        acc = None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(self.n, 3)
        t = np.ascontiguousarray(a_type, dtype=np.int32)
        m = np.ascontiguousarray(mass, dtype=np.float64)
        qq = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        mc = None if mic is None else np.ascontiguousarray(mic, dtype=np.int32).reshape(self.n, 3)
        ctx = C.c_void_p()
        check(self.lib.mfa_init(C.byref(self.params), precision, device, _dp(r0), _dp(v), _dp(acc),
                                _ip(t), _dp(m), _dp(qq), _ip(mc), C.byref(ctx)), "mfa_init")
        self.ctx = ctx
        self.mass = m
        self.a_type = t.copy()

    # ---- lifetime ----
    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.lib.mfa_finalize(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- the subroutines of md_main.f90:68-147 ----
    def set_step(self, i_time: int) -> None:
        check(self.lib.mfa_set_step(self.ctx, int(i_time)), "mfa_set_step")

    def verlet_positions(self) -> None:
        check(self.lib.mfa_verlet_positions(self.ctx), "verlet_positions")

    def check_skin(self) -> int:
        f = C.c_int32(0)
        check(self.lib.mfa_check_skin(self.ctx, C.byref(f)), "check_skin")
        return int(f.value)

    def binning(self) -> None:
        check(self.lib.mfa_binning(self.ctx), "binning")
        self.bin_type = 0

    def my_binning(self) -> None:
        check(self.lib.mfa_my_binning(self.ctx), "my_binning")
        self.bin_type = 1

    def rebuild(self) -> None:
        """The list rebuild of md_main.f90:81-85 with this system's rule."""
        if self.bin_type == 1:
            self.my_binning()
        else:
            self.binning()

    def zero_forces(self) -> None:
        check(self.lib.mfa_zero_forces(self.ctx), "zero_forces")

    def fluid_fluid(self) -> None:
        check(self.lib.mfa_fluid_fluid(self.ctx), "fluid_fluid")

    def pair_forces(self) -> None:
        """fluid_fluid and fluid_wall (WALL 2 fused) in one pass; adds to force."""
        check(self.lib.mfa_pair_forces(self.ctx), "pair_forces")

    def forces(self) -> None:
        """All forces of a step (fluid_fluid, fluid_wall, intra_molec, bending,
        ewald_k) in the fused passes of the time-step loop; adds to force."""
        check(self.lib.mfa_forces(self.ctx), "forces")

    def fluid_wall(self, inter_type: int) -> None:
        check(self.lib.mfa_fluid_wall(self.ctx, int(inter_type)), "fluid_wall")

    def intra_molec(self) -> None:
        check(self.lib.mfa_intra_molec(self.ctx), "intra_molec")

    def bending(self, mode: int) -> None:
        check(self.lib.mfa_bending(self.ctx, int(mode)), "bending")

    def ewald_k(self, mode: int) -> None:
        check(self.lib.mfa_ewald_k(self.ctx, int(mode)), "ewald_k")

    def dipolar_correction(self) -> None:
        check(self.lib.mfa_dipolar_correction(self.ctx), "dipolar_correction")

    def verlet_velocities(self) -> None:
        check(self.lib.mfa_verlet_velocities(self.ctx), "verlet_velocities")

    # ---- optional terms behind the reference's cpp switches ----
    def external_force(self, mode: int, k_elastic: float) -> None:
        """external_force(mode) (EXT_FORCE 1): elastic pull towards y = Ly/2, z = Lz/2."""
        check(self.lib.mfa_external_force(self.ctx, int(mode), float(k_elastic)), "external_force")

    def orientation(self, mode: int, k_or: float, alpha_or: float = 0.0, energy: bool = False):
        """orientation(mode) (ORIENTATION); returns v_or when energy=True (synchronises)."""
        out = C.c_double(0.0)
        check(self.lib.mfa_orientation(self.ctx, int(mode), float(k_or), float(alpha_or),
                                       C.byref(out) if energy else None), "orientation")
        return out.value if energy else None

    def set_dpd_vv(self, on: bool = True) -> None:
        """The DPD_VV switch: verlet_velocities becomes the kick alone, new_dpd_fd follows it."""
        check(self.lib.mfa_set_dpd_vv(self.ctx, int(bool(on))), "set_dpd_vv")
        self.dpd_vv = bool(on)

    def new_dpd_fd(self) -> None:
        check(self.lib.mfa_new_dpd_fd(self.ctx), "new_dpd_fd")

    # ---- compositions ----
    def init_forces(self, full: bool = False) -> None:
        """The start-up sequence of conf_default.f90:254-299: lists, the forces
        fluid_fluid / fluid_wall / intra_molec, then a = F/m.  full=True also
        adds bending and the Ewald k-space forces (the complete per-step force
        set), for starting a run from a state produced elsewhere."""
        p = self.params
        if p.charged:
            self.ewald_k(0)
        self.rebuild()
        self.zero_forces()
        self.fluid_fluid()
        if p.symmetry == 0 and p.wall in (2, 3, 4):
            self.fluid_wall(p.wall)
        self.intra_molec()
        if full and p.bending:
            self.bending(2)
        if full and p.charged:
            self.ewald_k(1)
            if p.symmetry == 0:
                self.dipolar_correction()
        f = self.download(_abi.F)["force"]
        self.upload(a=f / self.mass[:, None])

    def md_step(self) -> int:
        """One md_main.f90:68-147 iteration through the individual entry points.
        Returns f_skin as check_skin saw it."""
        p = self.params
        self.verlet_positions()
        f_skin = self.check_skin()
        if f_skin == 1:
            self.rebuild()
        self.zero_forces()
        self.fluid_fluid()
        if p.symmetry == 0 and p.wall in (2, 3, 4):
            self.fluid_wall(p.wall)
        self.intra_molec()
        if p.bending:
            self.bending(2)
        if p.charged:
            self.ewald_k(1)
            if p.symmetry == 0:
                self.dipolar_correction()     # md_main.f90:128-131
        self.verlet_velocities()
        if getattr(self, "dpd_vv", False):
            self.new_dpd_fd()                 # md_main.f90:149-155
        return f_skin

    def step(self, nsteps: int) -> None:
        """nsteps time steps on the device (fused kernels, captured graphs)."""
        check(self.lib.mfa_step(self.ctx, int(nsteps)), "mfa_step")

    def set_pair_queue(self, ctas_per_sm: int) -> None:
        """mfa_set_pair_queue: untiled pair launches with a work queue of
        ctas_per_sm CTAs per multiprocessor (0: one CTA per block of slots)."""
        check(self.lib.mfa_set_pair_queue(self.ctx, int(ctas_per_sm)), "mfa_set_pair_queue")

    def set_pair_split(self, pieces: int) -> None:
        """mfa_set_pair_split: untiled pair launches cut each 32-particle
        chunk's list into `pieces` runs, one warp each."""
        check(self.lib.mfa_set_pair_split(self.ctx, int(pieces)), "mfa_set_pair_split")

    def pair_split(self) -> int:
        """mfa_get_pair_split: the current pieces per chunk."""
        v = C.c_int32(0)
        check(self.lib.mfa_get_pair_split(self.ctx, C.byref(v)), "mfa_get_pair_split")
        return int(v.value)

    def set_pair_shape(self, entries_per_round: int, block: int, tiled: bool = True) -> None:
        check(self.lib.mfa_set_pair_shape(self.ctx, int(entries_per_round), int(block), int(bool(tiled))),
              "mfa_set_pair_shape")

    def set_cells(self, n_bin, skin: float) -> None:
        nb = (C.c_int32 * 3)(*[int(x) for x in n_bin])
        check(self.lib.mfa_set_cells(self.ctx, nb, float(skin)), "mfa_set_cells")
        self.params.skin = float(skin)
        for d in range(3):
            self.params.n_bin[d] = int(n_bin[d])

    # ---- trajectory sensitivities ----
    GRAD_NAMES = ("eps_lj", "sigma", "k_fene", "r0", "gamma_dpd", "eps_wall")

    def trajectory_observable(self, nsteps: int) -> float:
        """J = time average over nsteps steps of <z> + <R_ee^2> (the state advances)."""
        j = C.c_double(0.0)
        check(self.lib.mfa_trajectory_observable(self.ctx, int(nsteps), C.byref(j)), "mfa_trajectory_observable")
        return float(j.value)

    def adjoint(self, nsteps: int, every: int = 20):
        """(J, {parameter: dJ/dparameter}) by the hand-written adjoint (the state advances)."""
        out = (C.c_double * 7)()
        check(self.lib.mfa_adjoint(self.ctx, int(nsteps), int(every), out), "mfa_adjoint")
        return float(out[0]), {k: float(out[1 + i]) for i, k in enumerate(self.GRAD_NAMES)}

    # ---- mirrors ----
    def stream_ptr(self) -> int:
        """cudaStream_t of the context (for event timing on the launching stream)."""
        s = C.c_void_p()
        check(self.lib.mfa_stream(self.ctx, C.byref(s)), "mfa_stream")
        return int(s.value or 0)

    def sync(self) -> None:
        check(self.lib.mfa_sync(self.ctx), "mfa_sync")

    def scalars(self) -> dict:
        s = MfaScalars()
        check(self.lib.mfa_get_scalars(self.ctx, C.byref(s)), "mfa_get_scalars")
        return s.as_dict()

    def download(self, mask: int = _abi.R0 | _abi.V | _abi.A | _abi.F | _abi.MIC, out: dict | None = None) -> dict:
        """mfa_download of the quantities in mask.  `out` may hold the
        destination arrays (n x 3, C-contiguous; float64, int32 for mic) by
        name, e.g. pinned host buffers, which the device then writes directly."""
        n = self.n
        out = out or {}

        def dest(name, flag, dtype=np.float64):
            if not mask & flag:
                return None
            x = out.get(name)
            if x is None:
                return np.empty((n, 3), dtype=dtype)
            if x.shape != (n, 3) or x.dtype != dtype or not x.flags.c_contiguous:
                raise ValueError(f"download: {name} must be a C-contiguous ({n}, 3) {np.dtype(dtype).name} array")
            return x

        r0, v, a = dest("r0", _abi.R0), dest("v", _abi.V), dest("a", _abi.A)
        f = dest("force", _abi.F)
        mic = dest("mic", _abi.MIC, np.int32)
        check(self.lib.mfa_download(self.ctx, mask, _dp(r0), _dp(v), _dp(a), _dp(f), _ip(mic)),
              "mfa_download")
        return {"r0": r0, "v": v, "a": a, "force": f, "mic": mic}

    def upload(self, r0=None, v=None, a=None, force=None, mic=None) -> None:
        mask = 0
        arrs = []
        for bit, x, dt in ((_abi.R0, r0, np.float64), (_abi.V, v, np.float64), (_abi.A, a, np.float64),
                           (_abi.F, force, np.float64), (_abi.MIC, mic, np.int32)):
            if x is not None:
                mask |= bit
                arrs.append(np.ascontiguousarray(x, dtype=dt).reshape(self.n, 3))
            else:
                arrs.append(None)
        check(self.lib.mfa_upload(self.ctx, mask, _dp(arrs[0]), _dp(arrs[1]), _dp(arrs[2]),
                                  _dp(arrs[3]), _ip(arrs[4])), "mfa_upload")

    def debug_lists(self, max_per: int = 256):
        n = self.n
        cell = np.empty(n, dtype=np.int32)
        cnt = np.empty(n, dtype=np.int32)
        nbr = np.zeros((n, max_per), dtype=np.int32)
        check(self.lib.mfa_debug_lists(self.ctx, _ip(cell), _ip(cnt), _ip(nbr), max_per), "mfa_debug_lists")
        return cell, cnt, nbr

    def kvecs(self, max_k: int = 100000) -> np.ndarray:
        nk = C.c_int32(0)
        out = np.empty((max_k, 3))
        check(self.lib.mfa_debug_kvecs(self.ctx, C.byref(nk), _dp(out), max_k), "mfa_debug_kvecs")
        return out[: nk.value].copy()

    def observe(self) -> dict:
        """mfa_observe: radii of gyration (brush, melt) and total momentum."""
        o = _abi.MfaObservables()
        check(self.lib.mfa_observe(self.ctx, C.byref(o)), "mfa_observe")
        return {"r_g2_brush": np.array(o.r_g2_brush[:]), "r_g2_melt": np.array(o.r_g2_melt[:]),
                "momentum": np.array(o.momentum[:])}

    def observe_ends(self) -> dict:
        """mfa_observe_ends: mean end-to-end vectors and their squares for the
        top brushes, bottom brushes and melt (3 x 3 each), and minus the
        summed force on the heads of the upper- and lower-wall chains (2 x 3)."""
        ree, ree2, fh = np.empty(9), np.empty(9), np.empty(6)
        check(self.lib.mfa_observe_ends(self.ctx, _dp(ree), _dp(ree2), _dp(fh)), "mfa_observe_ends")
        return {"r_ee": ree.reshape(3, 3), "r_ee2": ree2.reshape(3, 3), "head_force": fh.reshape(2, 3)}

    def histogram_z(self, hist_dim: int, reset: bool = False):
        """mfa_histogram_z: adds this state's z histograms; returns the
        accumulated counts (2 x hist_dim: brush, melt) and observation count."""
        out = np.zeros((2, hist_dim))
        n = C.c_int32(0)
        check(self.lib.mfa_histogram_z(self.ctx, int(hist_dim), int(bool(reset)), _dp(out), C.byref(n)),
              "mfa_histogram_z")
        return out, n.value

    def density_profiles(self, counts, n_obs):
        """histo(1) normalisation (functions.f90:139): counts * hist_dim /
        (Lz * n_obs * Lx * Ly), with the bin centres."""
        L = np.asarray(self.params.boundary[:3], dtype=np.float64)
        hd = counts.shape[1]
        dens = counts * hd * (1.0 / L[2]) / (n_obs * (L[0] * L[1]))
        z = (np.arange(hd) + 0.5) * (L[2] / hd)
        return z, dens

    def set_energy_log(self, every: int, capacity: int) -> None:
        check(self.lib.mfa_set_energy_log(self.ctx, every, capacity), "mfa_set_energy_log")

    def energy_log(self, max_entries: int = 1 << 20) -> np.ndarray:
        out = np.empty((max_entries, 4))
        n = C.c_int32(0)
        check(self.lib.mfa_read_energy_log(self.ctx, _dp(out), max_entries, C.byref(n)), "mfa_read_energy_log")
        return out[: n.value].copy()

    def fetch_energy_log(self, out: np.ndarray, first: int, count: int) -> None:
        """mfa_fetch_energy_log: enqueue the copy of log entries
        [first, first + count) into ``out`` (a C-contiguous float64 array of at
        least count x 4, best in pinned memory) without waiting; ``out`` holds
        them after the next synchronising call (sync, scalars, download)."""
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size < 4 * count:
            raise ValueError("out: C-contiguous float64 array of at least count x 4 entries")
        check(self.lib.mfa_fetch_energy_log(self.ctx, _dp(out), first, count), "mfa_fetch_energy_log")


def from_config(cfg, precision: int = _abi.MIXED, device: int = 0) -> System:
    """A System holding a generated configuration (mfa_b200.configs)."""
    return System(cfg.params, cfg.r0, cfg.v, cfg.a_type, cfg.mass, q=cfg.q,
                  precision=precision, device=device)


class Batch:
    """Several Systems advanced together: each kernel stage of the time step is
    one launch for all of them (mfa_batch_*).  The Systems keep their state,
    energies and errors; read them after ``sync()``."""

    def __init__(self, systems):
        self.lib = load()
        self.systems = list(systems)
        arr = (C.c_void_p * len(self.systems))(*[s.ctx.value for s in self.systems])
        b = C.c_void_p()
        check(self.lib.mfa_batch_create(arr, len(self.systems), C.byref(b)), "mfa_batch_create")
        self.b = b

    def step(self, nsteps: int) -> None:
        check(self.lib.mfa_batch_step(self.b, int(nsteps)), "mfa_batch_step")

    def sync(self) -> None:
        check(self.lib.mfa_batch_sync(self.b), "mfa_batch_sync")

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        check(self.lib.mfa_batch_stream(self.b, C.byref(s)), "mfa_batch_stream")
        return int(s.value or 0)

    def launches(self) -> int:
        n = C.c_int64(0)
        check(self.lib.mfa_batch_launches(self.b, C.byref(n)), "mfa_batch_launches")
        return int(n.value)

    def scalars(self):
        """Per-system scalars (mfa_get_scalars of each system)."""
        self.sync()
        return [s.scalars() for s in self.systems]

    def close(self) -> None:
        if getattr(self, "b", None):
            self.lib.mfa_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
