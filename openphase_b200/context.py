"""`Context`: one device-resident phase-field state and its parameters, over the opgpu C ABI."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import FP32, FP64, STENCIL, Grid, Model, OpgpuError, Stats, lib, ptr


def _check(rc: int, h=None, what: str = ""):
    hard = rc & ~_lib.SOFT_MASK
    if hard:
        msg = lib().opgpu_last_error(h).decode() if h else ""
        raise OpgpuError(rc, f"{what}: {msg}")
    return rc


class Context:
    """Device state of one simulation (grid, K-slot field storage, grains, parameters)."""

    def __init__(self, nx, ny, nz, *, dx=1.0, iwidth=5.0, stencil="LB", gradient_stencil="ISOTROPIC",
                 precision="fp64", k_slots=8, device=0):
        L = lib()
        g = Grid(nx=nx, ny=ny, nz=nz, dx=dx, iwidth=iwidth, laplacian_stencil=STENCIL[stencil],
                 gradient_stencil=STENCIL[gradient_stencil], precision=FP32 if precision == "fp32" else FP64,
                 k_slots=k_slots, device=device)
        h = C.c_void_p()
        rc = L.opgpu_create(C.byref(g), C.byref(h))
        if rc:
            raise OpgpuError(rc, "opgpu_create")
        self.h = h
        self.shape = (nx, ny, nz)
        self.n = nx * ny * nz
        self.precision = precision
        self.k_slots = k_slots
        self.ngrains = 0

    def close(self):
        if getattr(self, "h", None):
            lib().opgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:   # interpreter shutdown: the library module may already be torn down
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- parameters
    def set_model(self, sigma, mu, *, limit=None, limiting=True, regularization=1.0, tj_factor=0.0,
                  consider_nucleus_volume=True, nucleus_volume_factor=1.0, energy_model=None, cubic_eps=None,
                  phase_solid=None, model_eps=None, facets=None, mobility_model=None, mobility_eps=None,
                  mobility_facets=None):
        """facets: (facet_start[P*P+1], facet_data[F, 5], facet_family[P*P]) of the FACETED and
        FACETEDEXP pairs; mobility_facets: the same for the FACETED mobility pairs."""
        sigma = np.ascontiguousarray(np.atleast_2d(sigma), dtype=np.float64)
        mu = np.ascontiguousarray(np.atleast_2d(mu), dtype=np.float64)
        lim = None if limit is None else np.ascontiguousarray(np.atleast_2d(limit), dtype=np.float64)
        em = None if energy_model is None else np.ascontiguousarray(energy_model, dtype=np.int32)
        eps = None if cubic_eps is None else np.ascontiguousarray(cubic_eps, dtype=np.float64)
        sol = None if phase_solid is None else np.ascontiguousarray(phase_solid, dtype=np.int32)
        meps = None if model_eps is None else np.ascontiguousarray(model_eps, dtype=np.float64)
        mm = None if mobility_model is None else np.ascontiguousarray(mobility_model, dtype=np.int32)
        mme = None if mobility_eps is None else np.ascontiguousarray(mobility_eps, dtype=np.float64)
        fs, fd, ff = (None, None, None) if facets is None else (
            np.ascontiguousarray(facets[0], dtype=np.int32), np.ascontiguousarray(facets[1], dtype=np.float64),
            np.ascontiguousarray(facets[2], dtype=np.int32))
        ms, md, mf = (None, None, None) if mobility_facets is None else (
            np.ascontiguousarray(mobility_facets[0], dtype=np.int32),
            np.ascontiguousarray(mobility_facets[1], dtype=np.float64),
            np.ascontiguousarray(mobility_facets[2], dtype=np.int32))
        as_ptr = lambda a, t: a.ctypes.data_as(C.POINTER(t)) if a is not None else None  # noqa: E731
        m = Model(nphases=sigma.shape[0], sigma=as_ptr(sigma, C.c_double), mu=as_ptr(mu, C.c_double),
                  limit=as_ptr(lim, C.c_double), limiting=int(limiting), regularization=regularization,
                  tj_factor=tj_factor, consider_nucleus_volume=int(consider_nucleus_volume),
                  nucleus_volume_factor=nucleus_volume_factor, energy_model=as_ptr(em, C.c_int32),
                  cubic_eps=as_ptr(eps, C.c_double), phase_solid=as_ptr(sol, C.c_int32),
                  model_eps=as_ptr(meps, C.c_double), facet_start=as_ptr(fs, C.c_int32),
                  facet_data=as_ptr(fd, C.c_double), facet_family=as_ptr(ff, C.c_int32),
                  mobility_model=as_ptr(mm, C.c_int32), mobility_eps=as_ptr(mme, C.c_double),
                  mobility_facet_start=as_ptr(ms, C.c_int32), mobility_facet_data=as_ptr(md, C.c_double),
                  mobility_facet_family=as_ptr(mf, C.c_int32))
        _check(lib().opgpu_set_model(self.h, C.byref(m)), self.h, "set_model")

    def set_averaging(self, enable: bool, range_: int = 0, threshold: float = 0.0):
        """DrivingForce $Average Yes/No (with $Range, $Threshold; 0 = the reference defaults)."""
        _check(lib().opgpu_set_averaging(self.h, int(enable), int(range_), float(threshold)), self.h, "set_averaging")

    def set_orientations(self, quat):
        q = None if quat is None else np.ascontiguousarray(quat, dtype=np.float64)
        _check(lib().opgpu_set_orientations(self.h, ptr(q)), self.h, "set_orientations")

    def set_grains(self, ngrains, phase=None, stage=None):
        ph = None if phase is None else np.ascontiguousarray(phase, dtype=np.int32)
        st = None if stage is None else np.ascontiguousarray(stage, dtype=np.int32)
        _check(lib().opgpu_set_grains(self.h, ngrains, ptr(ph), ptr(st)), self.h, "set_grains")
        self.ngrains = ngrains

    def set_pair_table(self, sigma=None, mu=None):
        s = None if sigma is None else np.ascontiguousarray(sigma, dtype=np.float64)
        m = None if mu is None else np.ascontiguousarray(mu, dtype=np.float64)
        _check(lib().opgpu_set_pair_table(self.h, ptr(s), ptr(m)), self.h, "set_pair_table")

    def set_pair_hash(self, seed, lo, span):
        _check(lib().opgpu_set_pair_hash(self.h, seed, lo, span), self.h, "set_pair_hash")

    def set_driving_force(self, dg: Optional[np.ndarray]):
        d = None if dg is None else np.ascontiguousarray(dg, dtype=np.float64)
        _check(lib().opgpu_set_driving_force(self.h, ptr(d)), self.h, "set_driving_force")

    # ---- state
    def upload(self, counts, idx, val):
        c = np.ascontiguousarray(counts, dtype=np.int32)
        i = np.ascontiguousarray(idx, dtype=np.int32)
        v = np.ascontiguousarray(val, dtype=np.float64)
        _check(lib().opgpu_upload_lists(self.h, ptr(c), ptr(i), ptr(v)), self.h, "upload_lists")

    def read_raw(self, path):
        _check(lib().opgpu_read_raw(self.h, str(path).encode()), self.h, "read_raw")

    def write_raw(self, path):
        _check(lib().opgpu_write_raw(self.h, str(path).encode()), self.h, "write_raw")

    def write_grains(self, path):
        """Grain records in the reference's restart format (GrainsProperties::Write)."""
        _check(lib().opgpu_write_grains(self.h, str(path).encode()), self.h, "write_grains")

    def read_grains(self, path):
        """Grain records from a restart file (GrainsProperties::Read); then finalize_initialization."""
        _check(lib().opgpu_read_grains(self.h, str(path).encode()), self.h, "read_grains")

    def write_restart(self, raw_path, grains_path):
        """PhaseField::Write(Settings, tStep): the raw state and the grain records."""
        self.write_raw(raw_path)
        self.write_grains(grains_path)

    def read_restart(self, raw_path, grains_path) -> int:
        """PhaseField::Read(Settings, BC, tStep): raw state, grain records, then Finalize."""
        self.read_raw(raw_path)
        self.read_grains(grains_path)
        return self.finalize_initialization()

    def write_vtk(self, path):
        """PhaseField::WriteVTK of the current state (.vts, ASCII)."""
        _check(lib().opgpu_write_vtk(self.h, str(path).encode()), self.h, "write_vtk")

    def finalize_initialization(self) -> int:
        return _check(lib().opgpu_finalize_initialization(self.h), self.h, "finalize_initialization")

    def step(self, dt, nsteps=1) -> int:
        return _check(lib().opgpu_step(self.h, dt, nsteps), self.h, "step")

    def step_async(self, dt, nsteps=1):
        _check(lib().opgpu_step_async(self.h, dt, nsteps), self.h, "step_async")

    def sync(self) -> int:
        return _check(lib().opgpu_sync(self.h), self.h, "sync")

    def total_entries(self) -> int:
        t = C.c_int64(0)
        _check(lib().opgpu_total_entries(self.h, C.byref(t)), self.h, "total_entries")
        return t.value

    def download(self, out=None):
        """Ragged host copy of the state: counts[N], then (index, value) pairs in voxel order.

        `out` may give (counts int32[N], idx int32[>= total], val float64[>= total]) arrays to fill,
        e.g. pinned host memory; the arrays returned are then views trimmed to the entry count."""
        total = self.total_entries()
        if out is None:
            counts = np.empty(self.n, dtype=np.int32)
            idx = np.empty(total, dtype=np.int32)
            val = np.empty(total, dtype=np.float64)
        else:
            counts, idx, val = out
            if (counts.dtype != np.int32 or idx.dtype != np.int32 or val.dtype != np.float64 or counts.size != self.n
                    or idx.size < total or val.size < total or not all(a.flags.c_contiguous for a in out)):
                raise ValueError("download: out must be contiguous int32[N], int32[>=total], float64[>=total]")
        _check(lib().opgpu_download_lists(self.h, ptr(counts), ptr(idx), ptr(val)), self.h, "download_lists")
        return counts, idx[:total], val[:total]

    def flags(self):
        f = np.empty(self.n, dtype=np.int8)
        _check(lib().opgpu_download_flags(self.h, ptr(f)), self.h, "download_flags")
        return f

    def flags_noalloc(self):
        """The flags through opgpu_download_flags_noalloc (no device allocation; grids up to 256^3)."""
        f = np.empty(self.n, dtype=np.int8)
        _check(lib().opgpu_download_flags_noalloc(self.h, ptr(f)), self.h, "download_flags_noalloc")
        return f

    def grains(self):
        G = self.ngrains
        vol, vr, mx = (np.empty(G) for _ in range(3))
        ex, st = np.empty(G, dtype=np.int32), np.empty(G, dtype=np.int32)
        _check(lib().opgpu_grains(self.h, ptr(vol), ptr(vr), ptr(mx), ptr(ex), ptr(st)), self.h, "grains")
        return {"volume": vol, "volume_ratio": vr, "max_volume": mx, "exist": ex, "stage": st}

    def stats(self) -> dict:
        s = Stats()
        _check(lib().opgpu_get_stats(self.h, C.byref(s)), self.h, "get_stats")
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def set_kernel_variant(self, variant: str):
        """'tiled' (production) or 'generic' (full-grid kernel, same arithmetic)."""
        code = {"tiled": 0, "generic": 1}[variant]
        _check(lib().opgpu_set_kernel_variant(self.h, code), self.h, "set_kernel_variant")

    def set_timing(self, enable: bool):
        _check(lib().opgpu_set_timing(self.h, int(enable)), self.h, "set_timing")

    def clear_status(self):
        _check(lib().opgpu_clear_status(self.h), self.h, "clear_status")

    @property
    def stream(self) -> int:
        return lib().opgpu_stream(self.h) or 0

    # ---- checkpoints, adjoint, tangent-linear model
    def checkpoint_reserve(self, nslots: int):
        _check(lib().opgpu_checkpoint_reserve(self.h, int(nslots)), self.h, "checkpoint_reserve")

    def checkpoint_save(self, slot: int):
        _check(lib().opgpu_checkpoint_save(self.h, int(slot)), self.h, "checkpoint_save")

    def step_save_input(self, dt, slot: int) -> int:
        """One step that leaves the state it started from in checkpoint `slot` (no state copy)."""
        return _check(lib().opgpu_step_save_input(self.h, dt, slot), self.h, "step_save_input")

    def checkpoint_load(self, slot: int):
        _check(lib().opgpu_checkpoint_load(self.h, int(slot)), self.h, "checkpoint_load")

    def adjoint_begin(self, dL_dV):
        w = np.ascontiguousarray(dL_dV, dtype=np.float64)
        _check(lib().opgpu_adjoint_begin(self.h, ptr(w)), self.h, "adjoint_begin")

    def adjoint_step(self, slot: int, dt: float) -> int:
        return _check(lib().opgpu_adjoint_step(self.h, int(slot), float(dt)), self.h, "adjoint_step")

    def adjoint_gradients(self):
        G = self.ngrains
        ds, dm, dd = np.empty((G, G)), np.empty((G, G)), np.empty(G)
        _check(lib().opgpu_adjoint_gradients(self.h, ptr(ds), ptr(dm), ptr(dd)), self.h, "adjoint_gradients")
        return ds, dm, dd

    def tlm_begin(self, dsigma=None, dmu=None, ddg=None):
        conv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        ds, dm, dd = conv(dsigma), conv(dmu), conv(ddg)
        _check(lib().opgpu_tlm_begin(self.h, ptr(ds), ptr(dm), ptr(dd)), self.h, "tlm_begin")

    def tlm_step(self, dt: float, nsteps: int = 1) -> int:
        return _check(lib().opgpu_tlm_step(self.h, float(dt), int(nsteps)), self.h, "tlm_step")

    def tlm_volumes(self):
        dV = np.empty(self.ngrains)
        _check(lib().opgpu_tlm_volumes(self.h, ptr(dV)), self.h, "tlm_volumes")
        return dV

    # ---- slab decomposition (device buffers are passed as raw device addresses)
    def set_volume_window(self, x0: int, x1: int):
        _check(lib().opgpu_set_volume_window(self.h, int(x0), int(x1)), self.h, "set_volume_window")

    def plane_bytes(self) -> int:
        return int(lib().opgpu_plane_bytes(self.h))

    def pack_plane(self, x: int, dev_ptr: int):
        _check(lib().opgpu_pack_plane(self.h, int(x), C.c_void_p(dev_ptr)), self.h, "pack_plane")

    def unpack_plane(self, x: int, dev_ptr: int):
        _check(lib().opgpu_unpack_plane(self.h, int(x), C.c_void_p(dev_ptr)), self.h, "unpack_plane")

    def set_stream_ordered(self, enable: bool):
        """Slab calls only enqueue on the context's stream; the caller orders its streams."""
        _check(lib().opgpu_set_stream_ordered(self.h, int(enable)), self.h, "set_stream_ordered")

    def volume_recount(self):
        _check(lib().opgpu_volume_recount(self.h), self.h, "volume_recount")

    def step_partial(self, dt: float) -> int:
        return _check(lib().opgpu_step_partial(self.h, float(dt)), self.h, "step_partial")

    def volume_accumulator(self, dev_ptr: int):
        _check(lib().opgpu_volume_accumulator(self.h, C.c_void_p(dev_ptr)), self.h, "volume_accumulator")

    def step_complete(self, dev_ptr: int, initial: bool = False) -> int:
        return _check(lib().opgpu_step_complete(self.h, C.c_void_p(dev_ptr), int(initial)), self.h, "step_complete")

    # ---- convenience
    @classmethod
    def from_case(cls, case, precision="fp64", k_slots=8, device=0, state=None, threads=0, restart=None):
        """A context holding the case's model, grains and parameters, and its initial state (or the
        state of restart = (raw_path, grains_path) written by write_restart or by the reference)."""
        ctx = cls(case.nx, case.ny, case.nz, dx=case.dx, iwidth=case.iwidth, stencil=case.stencil,
                  gradient_stencil=case.gradient_stencil, precision=precision, k_slots=k_slots, device=device)
        ctx.set_model(case.sigma_phase(), case.mu_phase(), limit=case.limit_phase(), limiting=case.limiting,
                      regularization=case.regularization, tj_factor=case.tj_factor,
                      energy_model=case.energy_models(), cubic_eps=case.cubic_eps(), phase_solid=case.solid_phase(),
                      model_eps=case.model_eps(), facets=case.facet_tables(),
                      mobility_model=case.mobility_models(), mobility_eps=case.mobility_eps_table(),
                      mobility_facets=case.mobility_facet_tables())
        ctx.set_grains(case.ngrains, phase=case.grain_phase())
        if case.orientations:
            ctx.set_orientations(case.quaternions())
        ps = case.pair_sigma()
        if ps is not None:
            ctx.set_pair_table(ps, None)
        ctx.set_driving_force(case.driving_force())
        if getattr(case, "average", False):
            ctx.set_averaging(True)
        if restart is not None:
            ctx.read_restart(*restart)
            return ctx
        counts, idx, val = state if state is not None else case.initial_state(threads)
        ctx.upload(counts, idx, val)
        ctx.finalize_initialization()
        return ctx
