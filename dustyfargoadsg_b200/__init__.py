"""dustyfargoadsg_b200 -- the gas time step of Dusty FARGO-ADSG (AlgoGas) on a
single NVIDIA B200, behind the C ABI of include/fargo_b200.h.

Python here is a thin binding over libfargo_b200.so for tests, benchmarks and
scripting; the step itself runs in the library's CUDA kernels.  The C host
(dustyfargoadsg_b200/host) and the reference's own main (through the AlgoGas
drop-in of host/algogas_dropin.c) use the same library.
"""
import ctypes as C
import os

import numpy as np

from . import _ffi
from ._ffi import (FB_F_ALL, FB_F_DENS, FB_F_ENERGY, FB_F_VRAD, FB_F_VTHETA, FbDustState, FbError,
                   FbParams, FbProfiles, FbState, FbStepReport, check, load)

__all__ = ["Disc", "Batch", "read_par", "select_device", "FbError", "load", "CONFIG_DIR"]

CONFIG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "configs")


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def select_device(device):
    """Make `device` current for the library's CUDA runtime (this thread)."""
    check(load().fb_select_device(int(device)), "fb_select_device")


def read_par(path, **overrides):
    """Parse a reference .par file (ReadVariables rules) into FbParams.

    PLANETCONFIG is resolved like the reference does (relative to the
    current directory) and, failing that, relative to the .par file.
    """
    lib = load()
    p = FbParams()
    check(lib.fb_params_read_par(C.byref(p), os.fsencode(path)), "fb_params_read_par(%s)" % path)
    cfg = p.planetconfig.decode()
    if cfg and not os.path.isabs(cfg) and not os.path.exists(cfg):
        alt = os.path.join(os.path.dirname(os.path.abspath(path)), cfg)
        if os.path.exists(alt):
            p.planetconfig = alt.encode()
    for key, val in overrides.items():
        if key == "planetconfig":
            val = os.fsencode(val)
        setattr(p, key, val)
    return p


class Disc:
    """One disc on the GPU: parameters, device context and host mirrors."""

    DUST_ARRAYS = ("r", "th", "vr", "vth", "l", "size", "stokes")

    def __init__(self, params, noise=0.0, seed=0, state=None, dust_seed=None, tuning=None, mode=None):
        """mode: the library build, "parity" or "fast" (default: FB_MODE, else parity)."""
        self.lib = load(mode)
        self.mode = self.lib.fb_mode
        if isinstance(params, (str, os.PathLike)):
            params = read_par(params)
        self.p = params
        if self.p.unsupported:
            raise FbError(-2, "Disc", self.lib.fb_unsupported_name(C.byref(self.p)).decode())
        self.nr, self.ns = self.p.nrad, self.p.nsec
        self.nf = (self.nr + 1) * self.ns
        self.ctx = C.c_void_p()
        check(self.lib.fb_create(C.byref(self.p), None, C.byref(self.ctx)), "fb_create")
        if tuning is not None:
            self.set_tuning(tuning)
        self.fields = {k: np.zeros(self.nf) for k in ("dens", "vrad", "vtheta", "energy")}
        self.prof = {k: np.zeros(self.nr) for k in
                     ("sigma_med", "sigma_inf", "energy_med", "vtheta_med", "vrad_med", "global_soundspeed")}
        self.st = FbState()
        for k, a in self.fields.items():
            setattr(self.st, k, _ptr(a))
        self.pr = FbProfiles(*[_ptr(self.prof[k]) for k in
                               ("sigma_med", "sigma_inf", "energy_med", "vtheta_med", "vrad_med",
                                "global_soundspeed")])
        self.npart = int(self.p.nbpart)
        if self.npart > 0:
            self.dust_arrays = {k: np.zeros(self.npart) for k in self.DUST_ARRAYS}
            self.dst = FbDustState()
            self.dst.n = self.npart
            for k, a in self.dust_arrays.items():
                setattr(self.dst, k, _ptr(a))
        if state is None:
            check(self.lib.fb_init_state(C.byref(self.p), self.ctx, float(noise), int(seed),
                                         C.byref(self.st), C.byref(self.pr)), "fb_init_state", self.ctx, self.lib)
        else:
            self.set_state(state)
            if self.npart > 0 and "pc_r" in state:
                self.set_dust(state)
            return
        check(self.lib.fb_upload(self.ctx, C.byref(self.st), C.byref(self.pr)), "fb_upload", self.ctx, self.lib)
        if self.p.mhd_lsa and self.p.nbturbmodes > 0:
            # the turbulent modes draw from the reference's global drand48
            # stream: seeded when the .par is read (Interpret.c:404-407),
            # reseeded and advanced by the initial noise when there is some
            draws = self.nr * self.ns if (noise or self.p.add_noise) else 0
            self.set_lsa_stream(self.lib.fb_rand48_state(int(seed), draws))
        if self.npart > 0:
            # InitDustSystem reseeds the stream (Dsys.c:173)
            check(self.lib.fb_init_dust(C.byref(self.p), self.ctx, int(seed if dust_seed is None else dust_seed),
                                        C.byref(self.dst)), "fb_init_dust", self.ctx, self.lib)
            check(self.lib.fb_dust_upload(self.ctx, C.byref(self.dst)), "fb_dust_upload", self.ctx, self.lib)

    # -- turbulent potential -------------------------------------------
    def lsa_stream(self):
        """48-bit drand48 state the turbulent modes draw from next."""
        x = C.c_ulonglong()
        check(self.lib.fb_lsa_stream(self.ctx, C.byref(x), 0), "fb_lsa_stream", self.ctx, self.lib)
        return x.value

    def set_lsa_stream(self, x):
        v = C.c_ulonglong(int(x))
        check(self.lib.fb_lsa_stream(self.ctx, C.byref(v), 1), "fb_lsa_stream", self.ctx, self.lib)

    # -- launch shapes --------------------------------------------------
    def set_tuning(self, tuning):
        """Apply launch shapes: a dict of fb_tuning fields, or a tuning table
        ({"iso"|"energy": {"NrxNs": entry}}) looked up for this grid."""
        entry = tuning
        if "iso" in tuning or "energy" in tuning:
            kind = "energy" if self.p.energy_equation else "iso"
            entry = tuning.get(kind, {}).get("%dx%d" % (self.p.nrad, self.p.nsec))
            if entry is None:
                return False
        t = _ffi.FbTuning(*[int(entry.get(f, 0)) for f in
                            ("cell_block", "azi_cells_per_thread", "rad_columns", "rad_rings", "azi_variant")])
        check(self.lib.fb_set_tuning(self.ctx, C.byref(t)), "fb_set_tuning", self.ctx, self.lib)
        return True

    def tuning(self):
        t = _ffi.FbTuning()
        check(self.lib.fb_get_tuning(self.ctx, C.byref(t)), "fb_get_tuning", self.ctx, self.lib)
        return {f: getattr(t, f) for f, _ in t._fields_}

    # -- particles ------------------------------------------------------
    def set_dust(self, state):
        """Upload particles: pc_r, pc_th, pc_vr, pc_vth, pc_size (+ pc_l,
        pc_stokes; pc_rng_x / pc_kicks / pc_carry for the random stream)."""
        for k in self.DUST_ARRAYS:
            key = "pc_" + k
            if key in state:
                self.dust_arrays[k][:] = np.asarray(state[key], dtype=np.float64)[: self.npart]
        if "pc_l" not in state:
            self.dust_arrays["l"][:] = self.dust_arrays["r"] * self.dust_arrays["vth"]
        self.dst.rng_x = int(state.get("pc_rng_x", self.dst.rng_x))
        self.dst.kicks = int(state.get("pc_kicks", 0))
        carry = state.get("pc_carry", (0.0, 0.0))
        self.dst.carry[0], self.dst.carry[1] = float(carry[0]), float(carry[1])
        self.dst.particles_mass = 0.0
        check(self.lib.fb_dust_upload(self.ctx, C.byref(self.dst)), "fb_dust_upload", self.ctx, self.lib)

    def dust(self):
        """Download the particles: {pc_r, ..., pc_stokes, pc_rng_x, pc_kicks}."""
        check(self.lib.fb_dust_download(self.ctx, C.byref(self.dst)), "fb_dust_download", self.ctx, self.lib)
        out = {"pc_" + k: v.copy() for k, v in self.dust_arrays.items()}
        out.update(pc_rng_x=int(self.dst.rng_x), pc_kicks=int(self.dst.kicks),
                   pc_carry=(self.dst.carry[0], self.dst.carry[1]))
        return out

    # -- state ----------------------------------------------------------
    def set_state(self, state):
        """Upload a state dict: fields (dens, vrad, vtheta, energy) of
        (nrad+1)*nsec doubles, profiles (SigmaMed, ...) and scalars."""
        for k in ("dens", "vrad", "vtheta", "energy"):
            if k in state:
                self.fields[k][:] = np.asarray(state[k], dtype=np.float64).ravel()[: self.nf]
        names = {"SigmaMed": "sigma_med", "SigmaInf": "sigma_inf", "EnergyMed": "energy_med",
                 "VthetaMed": "vtheta_med", "VradMed": "vrad_med", "GLOBAL_SoundSpeed": "global_soundspeed"}
        for src, dst in names.items():
            if src in state:
                self.prof[dst][:] = np.asarray(state[src], dtype=np.float64)[: self.nr]
        st = self.st
        st.physical_time = float(state.get("PhysicalTime", 0.0))
        st.physical_time_initial = float(state.get("PhysicalTimeInitial", 0.0))
        st.omega_frame = float(state.get("OmegaFrame", self.p.omegaframe))
        st.lost_mass = float(state.get("LostMass", 0.0))
        st.mindt = float(state.get("MINDT", self.p.mindt))
        st.maxdt = float(state.get("MAXDT", self.p.maxdt))
        for q in range(3):
            st.stardiscbarycenter_x[q] = float(np.asarray(state.get("stardiscbarycenter_x", [0, 0, 0]))[q])
            st.stardiscbarycenter_y[q] = float(np.asarray(state.get("stardiscbarycenter_y", [0, 0, 0]))[q])
        if "pl_x" in state:
            n = len(np.atleast_1d(state["pl_x"]))
            pl = st.planets
            pl.nb = n
            cfg = _ffi.FbPlanets()
            check(self.lib.fb_planets_read_cfg(C.byref(self.p), self.p.planetconfig, C.byref(cfg)),
                  "fb_planets_read_cfg")
            for q in range(n):
                pl.mass[q] = float(np.atleast_1d(state["pl_mass"])[q])
                pl.x[q] = float(np.atleast_1d(state["pl_x"])[q])
                pl.y[q] = float(np.atleast_1d(state["pl_y"])[q])
                pl.vx[q] = float(np.atleast_1d(state["pl_vx"])[q])
                pl.vy[q] = float(np.atleast_1d(state["pl_vy"])[q])
                pl.acc[q] = cfg.acc[q]
                pl.initial_mass[q] = cfg.initial_mass[q]
                pl.final_mass[q] = cfg.final_mass[q]
                pl.feeldisk[q] = cfg.feeldisk[q]
                pl.feelothers[q] = cfg.feelothers[q]
                pl.binary[q] = cfg.binary[q]
        check(self.lib.fb_upload(self.ctx, C.byref(self.st), C.byref(self.pr)), "fb_upload", self.ctx, self.lib)

    def step(self):
        """One DT (AlgoGas) on the device; returns the step report.

        A DT in which the reference's crash test fired (negative energy,
        SourceEuler.c:545-566) completes like the reference's and is not an
        error here: rep.status is then FB_ERR_NEGATIVE and rep.crashes,
        rep.crash_substeps and rep.crash_time say what happened
        (crash_state() gives the state at the first crash)."""
        rep = FbStepReport()
        rc = self.lib.fb_algogas(self.ctx, C.byref(rep))
        if rc != _ffi.FB_ERR_NEGATIVE:
            check(rc, "fb_algogas", self.ctx, self.lib)
        return rep

    def crash_state(self):
        """The state at the first crash (rings 0..nrad-1), what the reference
        writes as gas*999.dat: {dens, vrad, vtheta, energy, crash_time}."""
        n = self.nr * self.ns
        out = {k: np.zeros(n) for k in ("dens", "vrad", "vtheta", "energy")}
        st = FbState()
        for k, a in out.items():
            setattr(st, k, _ptr(a))
        t = C.c_double()
        check(self.lib.fb_download_crash(self.ctx, C.byref(st), C.byref(t)), "fb_download_crash", self.ctx, self.lib)
        out["crash_time"] = t.value
        return out

    def stage(self, stage, dt):
        check(self.lib.fb_stage(self.ctx, int(stage), float(dt)), "fb_stage", self.ctx, self.lib)

    def download(self, mask=FB_F_ALL):
        check(self.lib.fb_download(self.ctx, C.byref(self.st), C.c_uint(mask)), "fb_download", self.ctx, self.lib)
        out = {k: v.copy() for k, v in self.fields.items()}
        st = self.st
        out.update(PhysicalTime=st.physical_time, LostMass=st.lost_mass, MINDT=st.mindt, MAXDT=st.maxdt,
                   OmegaFrame=st.omega_frame)
        n = st.planets.nb
        for name in ("mass", "x", "y", "vx", "vy"):
            out["pl_" + name] = np.array([getattr(st.planets, name)[q] for q in range(n)])
        return out

    def kernel_launches(self):
        return int(self.lib.fb_kernel_launches(self.ctx))

    def profile(self, enable=True):
        check(self.lib.fb_profile(self.ctx, 1 if enable else 0), "fb_profile", self.ctx, self.lib)

    def profile_read(self):
        """{stage name: (device ms, launches)} accumulated since profile()."""
        out = {}
        n = self.lib.fb_profile_read(self.ctx, 0, None, None, None)
        for idx in range(n):
            name, ms, cnt = C.c_char_p(), C.c_double(), C.c_longlong()
            self.lib.fb_profile_read(self.ctx, idx, C.byref(name), C.byref(ms), C.byref(cnt))
            out[name.value.decode()] = (ms.value, cnt.value)
        return out

    def derived(self, which):
        out = np.zeros(self.nf)
        check(self.lib.fb_download_derived(self.ctx, int(which), _ptr(out)), "fb_download_derived", self.ctx, self.lib)
        return out

    def vortensity(self, field=False):
        """Azimuthal means of Sigma (per ring) and of the vortensity (per
        interface ring), and optionally the vortensity field."""
        sm, vm = np.zeros(self.nr), np.zeros(self.nr)
        f = np.zeros(self.nf) if field else None
        check(self.lib.fb_vortensity(self.ctx, _ptr(f) if field else None, _ptr(sm), _ptr(vm)),
              "fb_vortensity", self.ctx, self.lib)
        return (sm, vm, f) if field else (sm, vm)

    def diagnostics(self):
        m, p = C.c_double(), C.c_double()
        check(self.lib.fb_diagnostics(self.ctx, C.byref(m), C.byref(p)), "fb_diagnostics", self.ctx, self.lib)
        return m.value, p.value

    def close(self):
        if self.ctx:
            self.lib.fb_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Batch:
    """Several discs advanced one DT each by a single graph launch
    (fb_batch_*); the discs stay usable on their own."""

    def __init__(self, discs):
        self.discs = list(discs)
        self.lib = self.discs[0].lib
        if any(d.lib is not self.lib for d in self.discs):
            raise ValueError("the discs of a batch must use the same library build")
        n = len(self.discs)
        arr = (C.c_void_p * n)(*[d.ctx for d in self.discs])
        self.b = C.c_void_p()
        check(self.lib.fb_batch_create(arr, n, C.byref(self.b)), "fb_batch_create", None, self.lib)
        self.reps = (FbStepReport * n)()

    def step(self):
        """One DT of every disc; returns the per-disc step reports."""
        rc = self.lib.fb_batch_algogas(self.b, self.reps)
        if rc != _ffi.FB_ERR_NEGATIVE:  # a crash is reported per disc, as in Disc.step
            check(rc, "fb_batch_algogas", None, self.lib)
        return list(self.reps)

    def close(self):
        if self.b:
            self.lib.fb_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
