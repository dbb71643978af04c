"""Python host-side mirror of the reference's GridNode / Poisson call surface.

Thin ctypes binding of lib/libamr_b200.so (include/amr_b200.h).  Method
names follow the reference (grid/grid_node.h:46-80, poisson/poisson.h:44-69,
euler/hydro_driver.h); every numerical call runs CUDA kernels in the library.
There is no CPU fallback: when the library or a GPU is missing the
constructor raises.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libamr_b200.so")

PHYSICS_EULER = 0
PHYSICS_EULER_GRAVITY = 1
PHYSICS_ZTWD = 2
RECON_MINMOD = 0
RECON_PPM = 1
PREC_FP64 = 0
PREC_MIXED = 1
PREC_MIXED_SOLVE = 2

ERRORS = {
    -1: "AMR_ERR_ARG", -2: "AMR_ERR_CUDA", -3: "AMR_ERR_RANGE", -4: "AMR_ERR_NOCONVERGE",
    -5: "AMR_ERR_TIMEOUT", -6: "AMR_ERR_STATE", -7: "AMR_ERR_CAPACITY", -8: "AMR_ERR_NODEVICE",
}


class AmrConfig(ctypes.Structure):
    _fields_ = [
        ("bw", ctypes.c_int), ("nx", ctypes.c_int), ("nf", ctypes.c_int), ("physics", ctypes.c_int),
        ("precision", ctypes.c_int), ("z_reflect", ctypes.c_int), ("mirror_refine_y", ctypes.c_int),
        ("max_refine_level", ctypes.c_int), ("min_level", ctypes.c_int), ("min_grid_life", ctypes.c_int),
        ("max_bricks", ctypes.c_int), ("persistent_solve", ctypes.c_int), ("reconstruction", ctypes.c_int),
        ("grid_dim", ctypes.c_double), ("origin", ctypes.c_double * 3), ("minmod_theta", ctypes.c_double),
        ("cfl", ctypes.c_double), ("gamma", ctypes.c_double), ("rho_floor", ctypes.c_double),
        ("ei_floor", ctypes.c_double), ("maxdtinc", ctypes.c_double), ("grav_g", ctypes.c_double),
    ]


class BinaryHeader(ctypes.Structure):
    """Binary::write's root header (binary/binary.cpp:70-94)."""
    _fields_ = [(k, ctypes.c_double) for k in ("l1x", "h", "M1", "fill_factor", "n", "R1", "q", "a", "K1", "K2",
                                                "phi0_1", "phi0_2", "Omega", "phase", "Omega0")] + [
        ("accretor_type", ctypes.c_int), ("donor_type", ctypes.c_int), ("dummy", ctypes.c_ubyte)]


class AmrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "AMR_ERR"), code, msg))
        self.code = code


_lib = None


def load_library(path=LIB_PATH):
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError("libamr_b200.so not built (run 3d-eulerian-amr_b200/build.py): %s" % path)
        lib = ctypes.CDLL(path)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.amr_default_config.argtypes = [ctypes.POINTER(AmrConfig)]
        lib.amr_create.argtypes = [ctypes.POINTER(AmrConfig), ctypes.POINTER(P)]
        lib.amr_destroy.argtypes = [P]
        lib.amr_last_error.argtypes = [P]
        lib.amr_last_error.restype = ctypes.c_char_p
        lib.amr_init_root.argtypes = [P]
        lib.amr_load_tree.argtypes = [P, I, ip, ip, ip]
        lib.amr_num_bricks.argtypes = [P]
        lib.amr_get_tree.argtypes = [P, ip, ip, ip, ip, ip, ip, dp]
        lib.amr_refine_from_flags.argtypes = [P, ctypes.POINTER(ctypes.c_ubyte), I, ip]
        lib.amr_set_time.argtypes = [P, D]
        lib.amr_get_time.argtypes = [P]
        lib.amr_get_time.restype = D
        lib.amr_zone_count.argtypes = [P]
        lib.amr_zone_count.restype = ctypes.c_longlong
        for name in ("amr_upload_state", "amr_download_state", "amr_upload_poisson", "amr_download_poisson",
                     "amr_get_flow_off", "amr_set_flow_off"):
            if hasattr(lib, name):
                getattr(lib, name).argtypes = [P, dp]
        for name in ("amr_synchronize", "amr_enforce_boundaries", "amr_store", "amr_restore",
                     "amr_compute_fluxes", "amr_inject_from_children", "amr_poisson_set_source",
                     "amr_poisson_boundaries", "amr_compute_forces", "amr_store_phi", "amr_restore_phi",
                     "amr_restore_half_phi"):
            if hasattr(lib, name):
                getattr(lib, name).argtypes = [P]
        lib.amr_add_difs.argtypes = [P, D, D]
        lib.amr_max_dt.argtypes = [P, dp]
        lib.amr_check_for_refine.argtypes = [P, D, I, ip]
        lib.amr_state_max.argtypes = [P, I, dp]
        lib.amr_sub_step.argtypes = [P, D, D]
        lib.amr_fused_sub_step.argtypes = [P, D, D, I]
        lib.amr_hydro_step.argtypes = [P, D, D]
        lib.amr_get_stream.argtypes = [P, ctypes.POINTER(ctypes.c_void_p)]
        lib.amr_profile_enable.argtypes = [P, I]
        lib.amr_profile_reset.argtypes = [P]
        lib.amr_profile_get.argtypes = [P, I, dp, ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(ctypes.c_char_p)]
        lib.amr_stats.argtypes = [P, ctypes.POINTER(ctypes.c_longlong), ip, ip, ip]
        lib.amr_profile_units.argtypes = [P, I, ctypes.POINTER(ctypes.c_longlong)]
        lib.amr_launch_count.argtypes = [P, ctypes.POINTER(ctypes.c_longlong)]
        if hasattr(lib, "amr_vcycle"):
            lib.amr_vcycle.argtypes = [P, dp]
            lib.amr_poisson_solve.argtypes = [P, D, I, dp, ip]
            lib.amr_grav_step.argtypes = [P, D, D, D, I]
            lib.amr_graph_solve.argtypes = [P, D, I, dp, ip]
            lib.amr_graph_grav_step.argtypes = [P, D, D, I, dp]
        if hasattr(lib, "amr_ztwd_step"):
            lib.amr_ztwd_set_eos.argtypes = [P, P]
            lib.amr_ztwd_set_frame.argtypes = [P, D, D, D, D]
            lib.amr_ztwd_pot.argtypes = [P, I]
            lib.amr_ztwd_step.argtypes = [P, D, D, D, I, dp]
        if hasattr(lib, "amr_state_sum"):
            lib.amr_state_sum.argtypes = [P, I, dp]
            lib.amr_mass_sum.argtypes = [P, I, dp]
            lib.amr_sum_lz.argtypes = [P, dp]
            lib.amr_m1m2data.argtypes = [P, dp, dp]
        if hasattr(lib, "amr_write_checkpoint"):
            lib.amr_write_checkpoint.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(BinaryHeader), D]
            lib.amr_read_checkpoint.argtypes = [P, ctypes.c_char_p, ctypes.POINTER(BinaryHeader)]
            lib.amr_write_output.argtypes = [P, ctypes.c_char_p]
        if hasattr(lib, "amr_solve_phases"):
            lib.amr_solve_phases.argtypes = [P, dp, ctypes.POINTER(ctypes.c_longlong), dp, I]
            lib.amr_solve_last_ms.argtypes = [P, ctypes.POINTER(ctypes.c_float)]
            if hasattr(lib, "amr_solve_totals"):
                lib.amr_solve_totals.argtypes = [P, dp, ctypes.POINTER(ctypes.c_longlong)]
            if hasattr(lib, "amr_solve_phase_waits"):
                lib.amr_solve_phase_waits.argtypes = [P, dp, I, dp, ctypes.POINTER(ctypes.c_longlong)]
            if hasattr(lib, "amr_relax_passes"):
                lib.amr_relax_passes.argtypes = [P, ctypes.POINTER(ctypes.c_longlong), I]
            if hasattr(lib, "amr_set_wait_limit"):
                lib.amr_set_wait_limit.argtypes = [P, I]
            lib.amr_set_solve_layout.argtypes = [P, I, I]
            lib.amr_solve_relax_split.argtypes = [P, dp, ctypes.POINTER(ctypes.c_longlong),
                                                  ctypes.POINTER(ctypes.c_longlong)]
            lib.amr_get_solve_layout.argtypes = [P, ip, ip, ip, ip, ip]
            lib.amr_solve_relax_level_ms.argtypes = [P, dp, I]
            lib.amr_autotune_solve.argtypes = [P, D, I, I, dp, I, ip, ip]
        _lib = lib
    return _lib


def default_config(**kw):
    lib = load_library()
    cfg = AmrConfig()
    lib.amr_default_config(ctypes.byref(cfg))
    for k, v in kw.items():
        if k == "origin":
            for d in range(3):
                cfg.origin[d] = v[d]
        else:
            setattr(cfg, k, v)
    return cfg


def read_output(path):
    """Parse a file of amr_write_output: dict with time, per-brick level, loc,
    offset, age, child_mask, h, U [n, nf, nx, nx, nx] and phi [n, nx, nx, nx]
    (None without self-gravity)."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != b"AMRB200O":
        raise ValueError("not an amr_write_output file")
    nf, nx, bw, n, has_phi = np.frombuffer(data, np.int32, 5, 8)
    pos = 8 + 32
    time = float(np.frombuffer(data, np.float64, 1, pos)[0])
    pos += 8
    cells = nx * nx * nx
    out = {k: [] for k in ("level", "loc", "offset", "age", "child_mask", "h", "U", "phi")}
    for _ in range(n):
        rec = np.frombuffer(data, np.int32, 9, pos)
        pos += 36
        out["level"].append(rec[0])
        out["loc"].append(rec[1:4])
        out["offset"].append(rec[4:7])
        out["age"].append(rec[7])
        out["child_mask"].append(rec[8])
        out["h"].append(np.frombuffer(data, np.float64, 1, pos)[0])
        pos += 8
        out["U"].append(np.frombuffer(data, np.float64, nf * cells, pos).reshape(nf, nx, nx, nx))
        pos += 8 * nf * cells
        if has_phi:
            out["phi"].append(np.frombuffer(data, np.float64, cells, pos).reshape(nx, nx, nx))
            pos += 8 * cells
    if pos != len(data):
        raise ValueError("trailing bytes in %s" % path)
    res = {k: np.array(v) for k, v in out.items() if k != "phi"}
    res["phi"] = np.array(out["phi"]) if has_phi else None
    res["time"] = time
    res["bw"] = int(bw)
    return res


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class AMR:
    """One octree + device brick pool (amr_ctx)."""

    def __init__(self, **cfg_kw):
        self.lib = load_library()
        self.cfg = default_config(**cfg_kw)
        ptr = ctypes.c_void_p()
        rc = self.lib.amr_create(ctypes.byref(self.cfg), ctypes.byref(ptr))
        if rc != 0:
            raise AmrError(rc, "amr_create failed (no GPU, or bad config)")
        self.ctx = ptr
        self.bw, self.nx, self.nf = self.cfg.bw, self.cfg.nx, self.cfg.nf
        self.gnx = self.nx + 2 * self.bw
        self.pnx = self.nx + 2

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.amr_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise AmrError(rc, self.lib.amr_last_error(self.ctx).decode(errors="replace"))
        return rc

    # ---- octree -----------------------------------------------------------
    def init(self):
        self._check(self.lib.amr_init_root(self.ctx))

    def load_tree(self, level, loc, age=None):
        level = np.ascontiguousarray(level, np.int32)
        loc = np.ascontiguousarray(loc, np.int32).reshape(-1)
        agep = _iptr(np.ascontiguousarray(age, np.int32)) if age is not None else None
        if age is not None:
            self._age_keep = np.ascontiguousarray(age, np.int32)
            agep = _iptr(self._age_keep)
        self._check(self.lib.amr_load_tree(self.ctx, len(level), _iptr(level), _iptr(loc), agep))

    @property
    def nbricks(self):
        return self.lib.amr_num_bricks(self.ctx)

    def get_tree(self):
        n = self.nbricks
        t = dict(level=np.zeros(n, np.int32), loc=np.zeros((n, 3), np.int32), offset=np.zeros((n, 3), np.int32),
                 age=np.zeros(n, np.int32), child_mask=np.zeros(n, np.int32), refine_mask=np.zeros(n, np.int32),
                 h=np.zeros(n, np.float64))
        self._check(self.lib.amr_get_tree(self.ctx, _iptr(t["level"]), _iptr(t["loc"]), _iptr(t["offset"]),
                                          _iptr(t["age"]), _iptr(t["child_mask"]), _iptr(t["refine_mask"]),
                                          _dptr(t["h"])))
        return t

    def refine_from_flags(self, flags, clear=True):
        f = np.ascontiguousarray(flags, np.uint8).reshape(-1)
        ch = ctypes.c_int()
        self._check(self.lib.amr_refine_from_flags(self.ctx, f.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                                   int(clear), ctypes.byref(ch)))
        return bool(ch.value)

    def set_time(self, t):
        self._check(self.lib.amr_set_time(self.ctx, float(t)))

    def get_time(self):
        return self.lib.amr_get_time(self.ctx)

    def get_zone_cnt(self):
        return self.lib.amr_zone_count(self.ctx)

    # ---- state ------------------------------------------------------------
    def upload_state(self, U):
        U = np.ascontiguousarray(U, np.float64)
        assert U.shape == (self.nbricks, self.nf, self.gnx, self.gnx, self.gnx), U.shape
        self._check(self.lib.amr_upload_state(self.ctx, _dptr(U)))

    def download_state(self):
        U = np.zeros((self.nbricks, self.nf, self.gnx, self.gnx, self.gnx), np.float64)
        self._check(self.lib.amr_download_state(self.ctx, _dptr(U)))
        return U

    def upload_poisson(self, P):
        P = np.ascontiguousarray(P, np.float64)
        assert P.shape == (8, self.nbricks, self.pnx, self.pnx, self.pnx), P.shape
        self._check(self.lib.amr_upload_poisson(self.ctx, _dptr(P)))

    def download_poisson(self):
        P = np.zeros((8, self.nbricks, self.pnx, self.pnx, self.pnx), np.float64)
        self._check(self.lib.amr_download_poisson(self.ctx, _dptr(P)))
        return P

    def flow_off(self):
        fo = np.zeros(self.nf, np.float64)
        self._check(self.lib.amr_get_flow_off(self.ctx, _dptr(fo)))
        return fo

    def set_flow_off(self, fo):
        fo = np.ascontiguousarray(fo, np.float64)
        self._check(self.lib.amr_set_flow_off(self.ctx, _dptr(fo)))

    def synchronize(self):
        self._check(self.lib.amr_synchronize(self.ctx))

    # ---- GridNode call surface --------------------------------------------
    def enforce_boundaries(self):
        self._check(self.lib.amr_enforce_boundaries(self.ctx))

    def store(self):
        self._check(self.lib.amr_store(self.ctx))

    def restore(self):
        self._check(self.lib.amr_restore(self.ctx))

    def compute_fluxes(self):
        self._check(self.lib.amr_compute_fluxes(self.ctx))

    def add_difs(self, dt, beta):
        self._check(self.lib.amr_add_difs(self.ctx, float(dt), float(beta)))

    def inject_from_children(self):
        self._check(self.lib.amr_inject_from_children(self.ctx))

    def max_dt(self):
        v = ctypes.c_double()
        self._check(self.lib.amr_max_dt(self.ctx, ctypes.byref(v)))
        return v.value

    def check_for_refine(self, min_refine_density, clear=True):
        ch = ctypes.c_int()
        self._check(self.lib.amr_check_for_refine(self.ctx, float(min_refine_density), int(clear), ctypes.byref(ch)))
        return bool(ch.value)

    def state_max(self, field=0):
        v = ctypes.c_double()
        self._check(self.lib.amr_state_max(self.ctx, int(field), ctypes.byref(v)))
        return v.value

    def sub_step(self, dt, beta):
        self._check(self.lib.amr_sub_step(self.ctx, float(dt), float(beta)))

    def fused_sub_step(self, dt, beta, blocks_per_sm=0):
        self._check(self.lib.amr_fused_sub_step(self.ctx, float(dt), float(beta), int(blocks_per_sm)))

    def hydro_step(self, dt, min_refine_density):
        self._check(self.lib.amr_hydro_step(self.ctx, float(dt), float(min_refine_density)))

    # ---- instrumentation ----------------------------------------------------
    def stream_handle(self):
        s = ctypes.c_void_p()
        self._check(self.lib.amr_get_stream(self.ctx, ctypes.byref(s)))
        return s.value

    def profile(self, on=True):
        self._check(self.lib.amr_profile_enable(self.ctx, int(on)))

    def profile_reset(self):
        self._check(self.lib.amr_profile_reset(self.ctx))

    def profile_get(self):
        out = {}
        for cls in range(20):
            ms = ctypes.c_double()
            n = ctypes.c_longlong()
            name = ctypes.c_char_p()
            self._check(self.lib.amr_profile_get(self.ctx, cls, ctypes.byref(ms), ctypes.byref(n),
                                                 ctypes.byref(name)))
            u = ctypes.c_longlong()
            self._check(self.lib.amr_profile_units(self.ctx, cls, ctypes.byref(u)))
            out[name.value.decode()] = dict(ms=ms.value, launches=n.value, units=u.value)
        return out

    def launch_count(self):
        n = ctypes.c_longlong()
        self._check(self.lib.amr_launch_count(self.ctx, ctypes.byref(n)))
        return n.value

    def stats(self):
        rc = ctypes.c_longlong()
        hz, nb, ml = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.amr_stats(self.ctx, ctypes.byref(rc), ctypes.byref(hz), ctypes.byref(nb),
                                       ctypes.byref(ml)))
        return dict(relax_calls=rc.value, reflux_hazards=hz.value, nbricks=nb.value, max_level=ml.value)

    # ---- Poisson ------------------------------------------------------------
    def vcycle(self):
        v = ctypes.c_double()
        self._check(self.lib.amr_vcycle(self.ctx, ctypes.byref(v)))
        return v.value

    def poisson_solve(self, tol, max_cycles=1000):
        e = ctypes.c_double()
        n = ctypes.c_int()
        self._check(self.lib.amr_poisson_solve(self.ctx, float(tol), int(max_cycles), ctypes.byref(e),
                                               ctypes.byref(n)))
        return e.value, n.value

    def compute_forces(self):
        self._check(self.lib.amr_compute_forces(self.ctx))

    def poisson_boundaries(self):
        self._check(self.lib.amr_poisson_boundaries(self.ctx))

    def graph_solve(self, tol, max_cycles=1000):
        e = ctypes.c_double()
        n = ctypes.c_int()
        self._check(self.lib.amr_graph_solve(self.ctx, float(tol), int(max_cycles), ctypes.byref(e),
                                             ctypes.byref(n)))
        return e.value, n.value

    SOLVE_PHASES = ("source", "restrict", "phi_faces", "phi_edges", "phi_vertices", "init", "vcycle_down",
                    "dphi_faces", "relax_first", "relax", "coarse_correction", "retire", "forces", "adjust_force",
                    "error")

    def solve_phases(self):
        n = len(self.SOLVE_PHASES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        by = (ctypes.c_double * n)()
        self._check(self.lib.amr_solve_phases(self.ctx, ms, cnt, by, n))
        return {k: {"ms": ms[i], "count": cnt[i], "bytes": by[i]} for i, k in enumerate(self.SOLVE_PHASES)}

    def solve_phase_waits(self):
        """Barrier share of each phase class (ms) and the relaxation level-sum time."""
        n = len(self.SOLVE_PHASES)
        w = np.zeros(n)
        ls = ctypes.c_double()
        cnt = ctypes.c_longlong()
        self._check(self.lib.amr_solve_phase_waits(self.ctx, _dptr(w), n, ctypes.byref(ls), ctypes.byref(cnt)))
        out = {k: w[i] for i, k in enumerate(self.SOLVE_PHASES)}
        out["level_sum"] = ls.value
        out["level_sum_count"] = cnt.value
        return out

    def solve_totals(self):
        """(device ms, count) of the persistent solve launches of graph_solve."""
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        self._check(self.lib.amr_solve_totals(self.ctx, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def solve_relax_level_ms(self, n=16):
        """Block 0's ms in the persistent solve's relaxation loops per level."""
        ms = np.zeros(n)
        self._check(self.lib.amr_solve_relax_level_ms(self.ctx, _dptr(ms), n))
        return ms

    def solve_relax_split(self):
        """Block 0's view of the shared-memory relaxation loops: ms waiting
        for neighbours, computing, waiting for the decision, publishing;
        passes and sweeps."""
        ms = np.zeros(4)
        p, s = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.amr_solve_relax_split(self.ctx, _dptr(ms), ctypes.byref(p), ctypes.byref(s)))
        return {"wait_neighbours_ms": ms[0], "pass_ms": ms[1], "wait_decision_ms": ms[2], "publish_ms": ms[3],
                "passes": p.value, "sweeps": s.value}

    def set_solve_layout(self, layout, blocks_per_sm=0):
        self._check(self.lib.amr_set_solve_layout(self.ctx, int(layout), int(blocks_per_sm)))

    def solve_layout(self):
        """(layout, blocks per SM cap, threads per block, blocks, layouts of this brick size)"""
        v = [ctypes.c_int() for _ in range(5)]
        self._check(self.lib.amr_get_solve_layout(self.ctx, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def autotune_solve(self, tol, max_cycles=10000, reps=2):
        """Times the persistent solve in every layout and blocks-per-SM cap,
        keeps the fastest; returns (per-trial ms or None, best trial)."""
        ms = np.zeros(16)
        nt, best = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.amr_autotune_solve(self.ctx, float(tol), int(max_cycles), int(reps), _dptr(ms), 16,
                                                ctypes.byref(nt), ctypes.byref(best)))
        return [None if m < 0 else float(m) for m in ms[:nt.value]], best.value

    def set_wait_limit(self, polls):
        """Polls per bounded wait of the persistent solve (0: the default)."""
        self._check(self.lib.amr_set_wait_limit(self.ctx, int(polls)))

    def relax_passes(self, n=16):
        """Relaxation passes per level since the context started (every form)."""
        out = (ctypes.c_longlong * n)()
        self._check(self.lib.amr_relax_passes(self.ctx, out, n))
        return np.array(out[:], dtype=np.int64)

    def solve_last_ms(self):
        v = ctypes.c_float()
        self._check(self.lib.amr_solve_last_ms(self.ctx, ctypes.byref(v)))
        return v.value

    def graph_grav_step(self, tol, dynamic_range=1.0e6, step_index=0):
        dt = ctypes.c_double()
        self._check(self.lib.amr_graph_grav_step(self.ctx, float(tol), float(dynamic_range), int(step_index),
                                                 ctypes.byref(dt)))
        return dt.value

    def grav_step(self, dt, tol, dynamic_range=1.0e6, step_index=0):
        self._check(self.lib.amr_grav_step(self.ctx, float(dt), float(tol), float(dynamic_range),
                                           int(step_index)))

    # ---- ZTWD binary (AMR_PHYSICS_ZTWD) -------------------------------------
    def ztwd_set_eos(self, helm):
        """Table and code units of a helm.Helm context (kept alive here)."""
        self._helm = helm
        self._check(self.lib.amr_ztwd_set_eos(self.ctx, helm.ctx))

    def ztwd_set_frame(self, omega, omega0, fR=0.0, ftheta=0.0):
        self._check(self.lib.amr_ztwd_set_frame(self.ctx, float(omega), float(omega0), float(fR), float(ftheta)))

    def ztwd_pot(self, mode):
        """0 pot_to_grid, 1 pot_from_grid, 2 add_pot_et, 3 sub_pot_et (binary.cpp:825-936)."""
        self._check(self.lib.amr_ztwd_pot(self.ctx, int(mode)))

    def ztwd_step(self, dt, tol, dynamic_range=1.0e6, step_index=0):
        """BinaryDriver::step; returns the step taken (after MAXDTINC retries)."""
        used = ctypes.c_double()
        self._check(self.lib.amr_ztwd_step(self.ctx, float(dt), float(tol), float(dynamic_range), int(step_index),
                                           ctypes.byref(used)))
        return used.value

    # ---- checkpoints (X.*.chk of the reference) --------------------------------
    def write_checkpoint(self, path, header=None, refine_alpha=1.0):
        """header: a BinaryHeader for BINARY-build files, None otherwise."""
        hp = ctypes.byref(header) if header is not None else None
        self._check(self.lib.amr_write_checkpoint(self.ctx, os.fsencode(path), hp, float(refine_alpha)))

    def write_output(self, path):
        """Headless output (amr_write_output); read it back with read_output."""
        self._check(self.lib.amr_write_output(self.ctx, os.fsencode(path)))

    def read_checkpoint(self, path, binary=False):
        """Loads tree + state; returns the BinaryHeader when binary=True."""
        h = BinaryHeader() if binary else None
        self._check(self.lib.amr_read_checkpoint(self.ctx, os.fsencode(path), ctypes.byref(h) if binary else None))
        return h

    # ---- diagnostics ------------------------------------------------------------
    def state_sum(self, field=0):
        """GridNode::state_sum of one field: (sum u dV, its x, y, z moments)."""
        out = np.zeros(4)
        self._check(self.lib.amr_state_sum(self.ctx, int(field), _dptr(out)))
        return out

    def mass_sum(self, frac):
        """Binary::mass_sum: (mass, centre of mass x, y, z) of the accretor (0) or donor (1)."""
        out = np.zeros(4)
        self._check(self.lib.amr_mass_sum(self.ctx, int(frac), _dptr(out)))
        return out

    def sum_lz(self):
        out = np.zeros(1)
        self._check(self.lib.amr_sum_lz(self.ctx, _dptr(out)))
        return float(out[0])

    M1M2_FIELDS = ("m1", "m2", "mc", "js1", "js2", "jorb", "jc", "a", "q", "total_energy", "kinetic", "I1", "I2",
                   "Ic", "V1", "V2")

    def m1m2data(self):
        """Binary::M1M2data: (dict of the 16 scalars plus x1, xdot1, x2,
        xdot2 as 3-vectors, the L1 point as (phi_eff, x, y, z)), and the raw
        28-value array in the C ABI's order."""
        out = np.zeros(28)
        l1 = np.zeros(4)
        self._check(self.lib.amr_m1m2data(self.ctx, _dptr(out), _dptr(l1)))
        d = {k: float(out[i]) for i, k in enumerate(self.M1M2_FIELDS)}
        for i, k in enumerate(("x1", "xdot1", "x2", "xdot2")):
            d[k] = out[16 + 3 * i:19 + 3 * i].copy()
        d["l1"] = l1
        return d, out

