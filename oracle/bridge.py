"""TEST INFRASTRUCTURE ONLY — Python access to the checkers.

* `Oracle`        ctypes wrapper of liboracle.so, the C restatement of the reference step
* `run_reference` runs the unmodified reference (oracle/_ref/ref_driver, built from the reference
                  sources by oracle/Makefile) on a case and returns its dumped states

Only the tests, the smoke check and the bench's CPU-baseline / reference legs import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_DRIVER = HERE / "_ref" / "ref_driver"
STENCIL = {"SIMPLE": 0, "ISOTROPIC": 1, "LB": 2}

S_LIST_OVERFLOW, S_EMPTY_VOXEL, S_NORMALIZE_WARN, S_LIMITER_CAP = 1, 2, 4, 8


class OpParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_double), ("iwidth", C.c_double),
                ("stencil", C.c_int), ("gradient_stencil", C.c_int), ("nphases", C.c_int), ("ngrains", C.c_int),
                ("grain_phase", C.c_void_p), ("phase_solid", C.c_void_p), ("sigma_phase", C.c_void_p),
                ("mu_phase", C.c_void_p), ("energy_model", C.c_void_p), ("cubic_eps", C.c_void_p),
                ("model_eps", C.c_void_p), ("facet_start", C.c_void_p), ("facet_data", C.c_void_p),
                ("facet_family", C.c_void_p), ("mobility_model", C.c_void_p), ("mobility_eps", C.c_void_p),
                ("mobility_facet_start", C.c_void_p), ("mobility_facet_data", C.c_void_p),
                ("mobility_facet_family", C.c_void_p), ("quat", C.c_void_p), ("pair_sigma", C.c_void_p), ("pair_mu", C.c_void_p), ("dg", C.c_void_p),
                ("limiting", C.c_int), ("limit_phase", C.c_void_p), ("regularization", C.c_double),
                ("tj_factor", C.c_double), ("consider_nucleus_volume", C.c_int),
                ("nucleus_volume_factor", C.c_double), ("threads", C.c_int), ("average", C.c_int)]


_olib = None


def build_oracle():
    """Compile liboracle.so (and the reference build when the reference sources are present)."""
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True, env=env)


def oracle_lib():
    global _olib
    if _olib is None:
        if not ORACLE_LIB.exists():
            build_oracle()
        L = C.CDLL(str(ORACLE_LIB))
        L.op_create.restype = C.c_void_p
        L.op_create.argtypes = [C.POINTER(OpParams), C.c_int]
        L.op_destroy.argtypes = [C.c_void_p]
        L.op_load.restype = C.c_int
        L.op_load.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.op_finalize_initialization.argtypes = [C.c_void_p]
        L.op_step.restype = C.c_uint32
        L.op_step.argtypes = [C.c_void_p, C.c_double, C.c_int]
        L.op_total_entries.restype = C.c_long
        L.op_total_entries.argtypes = [C.c_void_p]
        L.op_get_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.op_get_flags.argtypes = [C.c_void_p, C.c_void_p]
        L.op_wide_count.restype = C.c_long
        L.op_wide_count.argtypes = [C.c_void_p]
        L.op_get_grains.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        L.op_set_grains.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        L.op_raw_counts.restype = C.c_long
        L.op_raw_counts.argtypes = [C.c_void_p, C.c_long, C.c_long, C.c_void_p]
        _olib = L
    return _olib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """The C restatement of the reference step, loaded with a case's initial state."""

    def __init__(self, case, counts, idx, val, cap=32, threads=0):
        L = oracle_lib()
        self._keep = []

        def keep(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a)
            self._keep.append(a)
            return a

        G = case.ngrains
        P = case.nphases
        sig = keep(case.sigma_phase())
        mu = keep(case.mu_phase())
        lim = keep(case.limit_phase())
        gph = keep(case.grain_phase().astype(np.int32))
        sol = keep(case.solid_phase().astype(np.int32))
        em = case.energy_models()
        em = keep(em.astype(np.int32)) if em is not None else None
        eps = case.cubic_eps()
        eps = keep(eps) if eps is not None else None
        meps = case.model_eps()
        meps = keep(meps) if meps is not None else None
        fac = case.facet_tables()
        fac = tuple(keep(x) for x in fac) if fac is not None else None
        mm = case.mobility_models()
        mm = keep(mm) if mm is not None else None
        mme = case.mobility_eps_table()
        mme = keep(mme) if mme is not None else None
        mfac = case.mobility_facet_tables()
        mfac = tuple(keep(x) for x in mfac) if mfac is not None else None
        quat = case.quaternions()
        quat = keep(quat.astype(np.float64)) if quat is not None else None
        ps = case.pair_sigma()
        ps = keep(ps.astype(np.float64)) if ps is not None else None
        dg = case.driving_force()
        dg = keep(dg) if dg is not None else None
        p = OpParams(nx=case.nx, ny=case.ny, nz=case.nz, dx=case.dx, iwidth=case.iwidth,
                     stencil=STENCIL[case.stencil], gradient_stencil=STENCIL[case.gradient_stencil],
                     nphases=P, ngrains=G, grain_phase=_p(gph).value, phase_solid=_p(sol).value,
                     sigma_phase=_p(sig).value, mu_phase=_p(mu).value,
                     energy_model=_p(em).value if em is not None else None,
                     cubic_eps=_p(eps).value if eps is not None else None,
                     model_eps=_p(meps).value if meps is not None else None,
                     facet_start=_p(fac[0]).value if fac else None, facet_data=_p(fac[1]).value if fac else None,
                     facet_family=_p(fac[2]).value if fac else None,
                     mobility_model=_p(mm).value if mm is not None else None,
                     mobility_eps=_p(mme).value if mme is not None else None,
                     mobility_facet_start=_p(mfac[0]).value if mfac else None,
                     mobility_facet_data=_p(mfac[1]).value if mfac else None,
                     mobility_facet_family=_p(mfac[2]).value if mfac else None,
                     quat=_p(quat).value if quat is not None else None, pair_sigma=_p(ps).value if ps is not None else None, pair_mu=None,
                     dg=_p(dg).value if dg is not None else None, limiting=int(case.limiting),
                     limit_phase=_p(lim).value, regularization=case.regularization, tj_factor=case.tj_factor,
                     consider_nucleus_volume=1, nucleus_volume_factor=1.0, threads=threads,
                     average=int(getattr(case, "average", False)))
        self.case = case
        self.h = L.op_create(C.byref(p), cap)
        if not self.h:
            raise RuntimeError("op_create failed")
        counts = np.ascontiguousarray(counts, dtype=np.int32)
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        if L.op_load(self.h, _p(counts), _p(idx), _p(val)) != 0:
            raise RuntimeError("op_load: list longer than the oracle capacity")
        L.op_finalize_initialization(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            oracle_lib().op_destroy(self.h)
            self.h = None

    def step(self, nsteps, dt=None):
        return int(oracle_lib().op_step(self.h, self.case.dt if dt is None else dt, nsteps))

    def state(self, positive_only=False):
        """Per-voxel lists (counts, idx, val).  Like the reference's Fields after Finalize they include
        the zero-valued candidate entries of CalculateDerivativesSR; positive_only drops them, which
        leaves exactly the stored fields of the CUDA path."""
        L = oracle_lib()
        n = self.case.n
        total = L.op_total_entries(self.h)
        counts = np.empty(n, dtype=np.int32)
        idx = np.empty(total, dtype=np.int32)
        val = np.empty(total, dtype=np.float64)
        L.op_get_state(self.h, _p(counts), _p(idx), _p(val))
        if positive_only:
            return positive_entries(counts, idx, val)
        return counts, idx, val

    def flags(self):
        f = np.empty(self.case.n, dtype=np.int8)
        oracle_lib().op_get_flags(self.h, _p(f))
        return f

    def wide_count(self):
        return int(oracle_lib().op_wide_count(self.h))

    def grains(self):
        G = self.case.ngrains
        vol, vr, mx = (np.empty(G) for _ in range(3))
        ex, st = np.empty(G, dtype=np.int32), np.empty(G, dtype=np.int32)
        oracle_lib().op_get_grains(self.h, _p(vol), _p(vr), _p(mx), _p(ex), _p(st))
        return {"volume": vol, "volume_ratio": vr, "max_volume": mx, "exist": ex, "stage": st}


def positive_entries(counts, idx, val):
    """Drop zero-valued entries from ragged lists, keeping the order of the rest."""
    keep = np.asarray(val) != 0.0
    vox = np.repeat(np.arange(counts.size), counts)
    new_counts = np.bincount(vox[keep], minlength=counts.size).astype(np.int32)
    return new_counts, np.asarray(idx)[keep], np.asarray(val)[keep]


def parse_raw(data: bytes):
    """Parse a raw PhaseField file (the reference's PhaseField::Write) into (dims, counts, idx, val);
    the per-voxel count walk runs in the oracle library (a Python loop takes minutes at 256^3)."""
    nx, ny, nz = (int(x) for x in np.frombuffer(data[:12], dtype=np.int32))
    words = np.frombuffer(data, dtype=np.uint64, offset=12)
    n = nx * ny * nz
    counts = np.empty(n, dtype=np.int32)
    used = oracle_lib().op_raw_counts(_p(words), words.size, n, _p(counts))
    if used != words.size:
        raise ValueError("raw file size does not match its counts")
    starts = np.zeros(n, dtype=np.int64)
    np.cumsum(1 + 2 * counts[:-1].astype(np.int64), out=starts[1:])
    total = int(counts.sum(dtype=np.int64))
    first = np.repeat(starts + 1, counts)
    rank = np.arange(total, dtype=np.int64) - np.repeat(np.cumsum(counts, dtype=np.int64) - counts, counts)
    entry_pos = first + 2 * rank
    idx = words[entry_pos].astype(np.int32)
    val = words[entry_pos + 1].view(np.float64).copy()
    return (nx, ny, nz), counts, idx, val


def reference_available() -> bool:
    return REF_DRIVER.exists()


def _case_text(case, workdir: Path, dump_steps, threads, nsteps=None, vtk_steps=(), restart_grains=None):
    P = case.nphases
    nsteps = max(dump_steps) if nsteps is None else nsteps
    lines = [f"nx {case.nx}", f"ny {case.ny}", f"nz {case.nz}", f"dx {case.dx!r}", f"iwidth {case.iwidth!r}",
             f"stencil {case.stencil}", f"dt {case.dt!r}", f"nsteps {nsteps}", f"nphases {P}",
             f"ngrains {case.ngrains}", f"limiting {int(case.limiting)}", f"average {int(case.average)}",
             f"regularization {case.regularization!r}", f"tj_factor {case.tj_factor!r}",
             "dump_steps " + " ".join(str(s) for s in dump_steps)]
    if vtk_steps:
        lines.append("vtk_steps " + " ".join(str(s) for s in vtk_steps))
    if restart_grains:
        lines.append(f"restart_grains_file {restart_grains}")
    sig, mu, lim, sol = case.sigma_phase(), case.mu_phase(), case.limit_phase(), case.solid_phase()
    eps = case.cubic_eps()
    for a in range(P):
        lines.append(f"phase_state {a} {'SOLID' if sol[a] else 'LIQUID'}")
        for b in range(a, P):
            lines += [f"sigma {a} {b} {float(sig[a, b])!r}", f"mu {a} {b} {float(mu[a, b])!r}",
                      f"limit {a} {b} {float(lim[a, b])!r}"]
            if case.disorientation:
                lines.append(f"energy_model {a} {b} DISORIENTATION")
            elif case.facets and eps is not None and eps[a, b] != 0.0:
                lines.append(f"energy_model {a} {b} {'FACETEDEXP' if case.facet_exp else 'FACETED'}")
                lines.append(f"facet_family {a} {b} {int(case.facet_families)}")
                for (h, k, l, sf, ef) in case.facets:
                    lines.append(f"facet {a} {b} {h} {k} {l} {float(sf)!r} {float(ef)!r}")
            elif eps is not None and eps[a, b] != 0.0:
                name = case.hex_model or "CUBIC"
                lines += [f"energy_model {a} {b} {name}", f"cubic_eps {a} {b} {float(eps[a, b])!r}"]
                if case.hex_model:
                    lines.append(f"model_eps {a} {b} " + " ".join(repr(float(e)) for e in case.model_eps()[a, b]))
    mm = case.mobility_models()
    if mm is not None:
        for a in range(P):
            for b in range(a, P):
                if mm[a, b]:
                    lines.append(f"mobility_model {a} {b} {case.mobility_model}")
                    lines.append(f"mobility_eps {a} {b} " + " ".join(repr(float(e)) for e in case.mobility_eps))
                    if case.mobility_model == "FACETED":
                        lines.append(f"mobility_facet_family {a} {b} {int(case.mobility_facet_families)}")
                        for (h, k, l, mf, ef) in case.mobility_facets:
                            lines.append(f"mobility_facet {a} {b} {h} {k} {l} {float(mf)!r} {float(ef)!r}")
    if P > 1:
        f = workdir / "grain_phase.bin"
        case.grain_phase().astype(np.int32).tofile(f)
        lines.append(f"grain_phase_file {f}")
    quat = case.quaternions()
    if quat is not None:
        f = workdir / "orientation.bin"
        np.ascontiguousarray(quat, dtype=np.float64).tofile(f)
        lines.append(f"orientation_file {f}")
    if threads:
        lines.append(f"threads {threads}")
    ps = case.pair_sigma()
    if ps is not None:
        f = workdir / "pair_sigma.bin"
        np.ascontiguousarray(ps, dtype=np.float64).tofile(f)
        lines.append(f"pair_sigma_file {f}")
    dg = case.driving_force()
    if dg is not None:
        f = workdir / "dg.bin"
        dg.astype(np.float64).tofile(f)
        lines.append(f"dg_file {f}")
    return "\n".join(lines) + "\n"


def run_reference(case, counts, idx, val, dump_steps, threads=0, workdir=None, nsteps=None, proc_bind="close",
                  vtk_steps=(), restart_grains=None, keep_files=False):
    """Run the compiled reference on the case; returns {step: (counts, idx, val, volume, volume_ratio)}
    and the stats dictionary (wall time of the step loop, threads, wide-interface counts).

    nsteps defaults to the last dump step (dump_steps may then be empty); the OpenMP threads are
    bound with OMP_PROC_BIND=proc_bind.  vtk_steps: steps at which the reference writes its VTK file
    (returned as bytes under stats["vtk"][step]); restart_grains: a grain-record file to restart from
    (the reference's PhaseField::Read + FieldsProperties.Read + Finalize).  Each dumped step also
    carries the reference's grain-record file bytes under stats["grains_file"][step]."""
    from openphase_b200.initializations import raw_bytes

    if not REF_DRIVER.exists():
        raise FileNotFoundError("reference driver not built (make -C oracle ref)")
    tmp = tempfile.TemporaryDirectory() if workdir is None else None
    wd = Path(workdir or tmp.name)
    wd.mkdir(parents=True, exist_ok=True)
    (wd / "case.txt").write_text(_case_text(case, wd, dump_steps, threads, nsteps, vtk_steps, restart_grains))
    (wd / "init.dat").write_bytes(raw_bytes(case.nx, case.ny, case.nz, counts, idx, val))
    out = wd / "out"
    out.mkdir(exist_ok=True)
    env = dict(os.environ)
    if proc_bind:
        env["OMP_PROC_BIND"] = proc_bind
    r = subprocess.run([str(REF_DRIVER), str(wd / "case.txt"), str(wd / "init.dat"), str(out)],
                       capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"ref_driver failed ({r.returncode}): {r.stderr[-2000:]}")
    res = {}
    for s in dump_steps:
        _, c, i, v = parse_raw((out / f"PF_{s}.dat").read_bytes())
        vol = np.fromfile(out / f"V_{s}.bin", dtype=np.float64)
        vr = np.fromfile(out / f"VR_{s}.bin", dtype=np.float64)
        res[s] = (c, i, v, vol, vr)
    stats = {}
    for line in (out / "stats.txt").read_text().splitlines():
        k, *vals = line.split()
        stats[k] = [float(x) for x in vals] if len(vals) > 1 else float(vals[0])
    stats["vtk"] = {}
    for st in vtk_steps:
        files = sorted(out.glob(f"PhaseField_*{st}.vts"))
        files = [f for f in files if int(f.stem.split("_")[-1]) == st]
        stats["vtk"][st] = files[0].read_bytes()
    stats["grains_file"] = {st: (out / f"FP_{st}.dat").read_bytes() for st in dump_steps}
    if tmp is not None:
        tmp.cleanup()
    return res, stats
