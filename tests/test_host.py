"""CPU tests: the C ABI loads, the .par reader follows the reference's rules,
and the host-side initial state is bit-identical to the reference's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from tests import _oracle

REPO = _oracle.REPO
CFG = _oracle.CONFIG_DIR


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_library_exports_every_declared_symbol(mode):
    from dustyfargoadsg_b200 import _ffi
    lib = _ffi.load(mode)
    header = open(os.path.join(REPO, "include", "fargo_b200.h")).read()
    declared = set(re.findall(r"\b(fb_[a-z0-9_]+)\s*\(", header))
    assert declared, "no declarations parsed"
    for name in sorted(declared):
        assert hasattr(lib, name), name
    assert set(_ffi.EXPORTS) == declared
    info = lib.fb_build_info()
    assert b"sm_100a" in info
    assert (b"--fmad=true" in info) == (mode == "fast")


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_struct_layout_matches_ctypes(mode):
    from dustyfargoadsg_b200 import _ffi
    _ffi.check_layout(_ffi.load(mode))


def test_params_defaults_and_switches():
    from dustyfargoadsg_b200 import read_par
    p = read_par(os.path.join(CFG, "iso_128x384.par"))
    assert (p.nrad, p.nsec) == (128, 384)
    assert p.log_grid == 1 and p.fast_transport == 1 and p.wall_boundary == 1
    assert p.evanescent == 1 and abs(p.wkzrmin - 0.5) < 1e-15
    assert p.forced_circular == 1 and p.energy_equation == 0
    assert p.unsupported == 0
    assert abs(p.densityfloor - 1e-9) < 1e-24 and p.add_floors == 1
    assert p.masstaper == 0.0000001 and p.mindt == 100.0


def test_unsupported_features_are_refused(tmp_path):
    from dustyfargoadsg_b200 import Disc, FbError, read_par
    src = os.path.join(CFG, "iso_128x384.par")
    for keys in ({"InnerBoundary": "Accreting"}, {"Frame": "G"}, {"DustFluid": "Yes"},
                 {"EnergyEquation": "Yes", "RadiativeDiffusion": "Implicit", "Nsec": "385"}):
        key = ",".join(keys)
        par = _oracle.write_par(src, str(tmp_path), **keys)
        p = read_par(par)
        assert p.unsupported != 0, key
        with pytest.raises(FbError):
            Disc(p)


@pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")
@pytest.mark.parametrize("noise,seed,keys", [(0.0, 0, {}), (1e-4, 0, {}), (1e-3, 7, {}),
                                             (0.0, 5, {"AddNoise": "Yes", "Frame": "C"}),
                                             (1e-3, 3, {"AddNoise": "Yes", "Frame": "C", "ForcedCircular": "No"})])
def test_initial_state_bit_identical(tmp_path, noise, seed, keys):
    """fb_init_state == the reference's main.c initialisation, bit for bit,
    also with the reference's own AddNoise perturbation (seeded) and in the
    frame corotating with the planet (OmegaFrame from its orbit)."""
    from dustyfargoadsg_b200 import _ffi, read_par
    src = os.path.join(CFG, "iso_128x384.par")
    par = _oracle.write_par(src, str(tmp_path), Nrad=48, Nsec=96, **keys)
    dumps, _, _ = _oracle.run_oracle(par, steps=1, noise=noise, seed=seed, dump_every=1000)
    ref = dumps["state_init"]
    lib = _ffi.load()
    p = read_par(par)
    nr, ns = p.nrad, p.nsec
    nf = (nr + 1) * ns
    f = {k: np.zeros(nf) for k in ("dens", "vrad", "vtheta", "energy")}
    pr = {k: np.zeros(nr) for k in ("sigma_med", "sigma_inf", "energy_med", "vtheta_med", "vrad_med",
                                    "global_soundspeed")}
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    st = _ffi.FbState()
    for k, a in f.items():
        setattr(st, k, ptr(a))
    prof = _ffi.FbProfiles(*[ptr(pr[k]) for k in ("sigma_med", "sigma_inf", "energy_med", "vtheta_med",
                                                   "vrad_med", "global_soundspeed")])
    _ffi.check(lib.fb_init_state(C.byref(p), None, noise, seed, C.byref(st), C.byref(prof)), "init")
    for k in ("dens", "vrad", "vtheta", "energy"):
        np.testing.assert_array_equal(f[k], ref[k], err_msg=k)
    np.testing.assert_array_equal(pr["sigma_med"], ref["SigmaMed"])
    np.testing.assert_array_equal(pr["vtheta_med"], ref["VthetaMed"])
    np.testing.assert_array_equal(pr["vrad_med"], ref["VradMed"])
    np.testing.assert_array_equal(pr["global_soundspeed"], ref["GLOBAL_SoundSpeed"])
    assert st.planets.nb == 1
    assert st.planets.x[0] == ref["pl_x"][0] and st.planets.vy[0] == ref["pl_vy"][0]
    assert st.planets.mass[0] == ref["pl_mass"][0]
    assert st.omega_frame == ref["OmegaFrame"]


DUST_PAR = os.path.join(CFG, "dust_256x768.par")


@pytest.mark.skipif(not _oracle.have_oracle(), reason="oracle not built")
@pytest.mark.parametrize("keys", [
    dict(),                                                   # s^-3.5 sizes, uniform radii
    dict(SizePartSlope=1.0, DustSlope=1.0, SizeMaxPart=1e-1),  # the exp/log branches of Dsys.c:182-197
    dict(SizeMinPart=1e-3, SizeMaxPart=1e-3, SizePartSlope=0.0, DustSlope=0.5, RminDust=0.0),
])
def test_initial_particles_bit_identical(tmp_path, keys):
    """fb_init_dust == InitDustSystem (Dsys.c:128-262) bit for bit, and the
    drand48 stream is left at the same position."""
    from dustyfargoadsg_b200 import _ffi, read_par
    args = dict(Nrad=32, Nsec=64, NbPart=3000)
    args.update(keys)
    par = _oracle.write_par(DUST_PAR, str(tmp_path), **args)
    dumps, _, _ = _oracle.run_oracle(par, steps=1, noise=0.0, seed=1, dump_every=1000)
    ref = dumps["state_init"]
    lib = _ffi.load()
    p = read_par(par)
    assert p.unsupported == 0, lib.fb_unsupported_name(C.byref(p))
    n = p.nbpart
    arrays = {k: np.zeros(n) for k in ("r", "th", "vr", "vth", "l", "size", "stokes")}
    st = _ffi.FbDustState()
    st.n = n
    for k, a in arrays.items():
        setattr(st, k, a.ctypes.data_as(C.POINTER(C.c_double)))
    _ffi.check(lib.fb_init_dust(C.byref(p), None, 1, C.byref(st)), "fb_init_dust")
    for k in ("r", "th", "vr", "vth", "size"):
        np.testing.assert_array_equal(arrays[k], ref["pc_" + k], err_msg=k)
    np.testing.assert_array_equal(arrays["l"], arrays["r"] * arrays["vth"])
    assert st.rng_x == int(ref["rng_state"])
    assert st.kicks == 0


def test_inner_boundary_switches():
    """INNERBOUNDARY by first letter (src/Interpret.c:168-175): W wall, O open,
    K Kley & Nelson open, N non-reflecting; A (accreting) is refused."""
    import tempfile

    from dustyfargoadsg_b200 import read_par
    src = os.path.join(CFG, "iso_128x384.par")
    want = {"Wall": (1, 0, 0, 0), "Open": (0, 1, 0, 0), "KNOpen": (0, 1, 1, 0), "Non-Reflecting": (0, 0, 0, 1)}
    with tempfile.TemporaryDirectory() as wd:
        for val, flags in want.items():
            p = read_par(_oracle.write_par(src, wd, InnerBoundary=val))
            assert (p.wall_boundary, p.open_inner, p.kn_open, p.non_reflecting) == flags, val
            assert p.unsupported == 0, val


def test_turbulent_potential_parameters(tmp_path):
    """MHD L reads the turbulent potential's keys (src/var.c:99-102, 133-134)
    and is refused together with particles, whose kicks share the reference's
    drand48 stream with the modes."""
    from dustyfargoadsg_b200 import read_par
    lsa = dict(MHD="L", NbTurbModes="40", GammaTurb="2e-3", TurbRmin="0.6", TurbRmax="2.0", HighMCutoff="Yes")
    p = read_par(_oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par"), str(tmp_path), **lsa))
    assert p.unsupported == 0 and p.mhd_lsa == 1 and p.nbturbmodes == 40 and p.high_m_cutoff == 1
    assert p.gammaturb == 2e-3 and p.turbrmin == 0.6 and p.turbrmax == 2.0 and p.lsamodespeedup == 0.1
    os.makedirs(str(tmp_path / "d"))
    d = read_par(_oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "dust_256x768.par"), str(tmp_path / "d"),
                                   NbPart=100, **lsa))
    assert d.unsupported != 0
    os.makedirs(str(tmp_path / "m"))
    m = read_par(_oracle.write_par(os.path.join(_oracle.CONFIG_DIR, "iso_128x384.par"), str(tmp_path / "m"),
                                   **dict(lsa, NbTurbModes="1000")))
    assert m.unsupported != 0


def test_rand48_state_helper():
    """fb_rand48_state is srand48(seed) advanced by `draws` drand48 calls."""
    from dustyfargoadsg_b200 import load
    lib = load()
    x = (7 << 16) | 0x330E
    for _ in range(1000):
        x = (0x5DEECE66D * x + 0xB) & ((1 << 48) - 1)
    assert lib.fb_rand48_state(7, 1000) == x
    assert lib.fb_rand48_state(0, 0) == 0x330E


def test_thermal_diffusion_parameters(tmp_path):
    """ENTROPYDIFFUSION, RADIATIVEDIFFUSION (E explicit, I implicit) and
    DIFFUSIVITY (src/var.c:85-93, src/Interpret.c:381-388)."""
    from dustyfargoadsg_b200 import read_par
    src = os.path.join(CFG, "adiabatic_sg_512x1536.par")
    p = read_par(_oracle.write_par(src, str(tmp_path), EntropyDiffusion="Yes", Diffusivity="2e-5",
                                   RadiativeDiffusion="Explicit"))
    assert p.entropy_diffusion == 1 and p.radiative_diffusion == 1 and p.diffusivity == 2e-5 and p.unsupported == 0
    os.makedirs(str(tmp_path / "i"))
    q = read_par(_oracle.write_par(src, str(tmp_path / "i"), RadiativeDiffusion="Implicit"))
    assert q.radiative_diffusion == 2 and q.entropy_diffusion == 0 and q.diffusivity == 1e-6 and q.unsupported == 0


REF_IN = os.path.join(os.environ.get("FB_REFERENCE_DIR", os.path.join(os.path.dirname(REPO), "reference")), "in")


@pytest.mark.skipif(not os.path.isdir(REF_IN), reason="the reference's example parameter files are not here")
def test_reference_example_parameter_files_are_accepted():
    """Every example parameter file the reference ships (in/*.par: a
    corotating disc with non-reflecting edges, its energy-equation variant,
    the gas-only one, and the self-gravitating disc with AddNoise and
    TempPresc) is accepted as it is: no feature it sets is refused."""
    from dustyfargoadsg_b200 import _ffi, read_par
    lib = _ffi.load()
    pars = sorted(f for f in os.listdir(REF_IN) if f.endswith(".par"))
    assert pars
    for f in pars:
        p = read_par(os.path.join(REF_IN, f))
        assert p.unsupported == 0, (f, lib.fb_unsupported_name(C.byref(p)).decode())
