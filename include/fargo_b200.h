/*
 * fargo_b200.h -- C ABI of libfargo_b200.so, a B200 (sm_100a) implementation
 * of the gas time step of Dusty FARGO-ADSG.
 *
 * The boundary replaced is the reference's
 *     void AlgoGas(Force*, PolarGrid *Rho, *Vrad, *Vtheta, *Energy, *Label,
 *                  PolarGrid *DRho, *dustpcdens, *DVrad, *DVtheta,
 *                  PlanetarySystem*, DustSystem*)
 * (src/SourceEuler.c:326-331, prototype src/proto.h:82), called once per DT
 * from src/main.c:387.  Here the state lives on the GPU between calls;
 * the host uploads it once, calls fb_algogas() once per DT and downloads
 * fields only when it writes outputs.
 *
 * Conventions
 *  - Every entry point returns FB_OK (0) or a negative FB_ERR_* code.  The
 *    library never calls exit(); fb_last_error() gives a one-line reason.
 *  - Fields use the reference's PolarGrid layout: ring-major, index
 *    l = j + i*nsec, with nrad+1 rings (ring nrad holds the outer radial
 *    velocity interface, src/LowTasks.c:97-112).  Host buffers passed to
 *    fb_upload / fb_download have (nrad+1)*nsec doubles.
 *  - FP64 throughout.  A context is not thread-safe; use one per host thread.
 *  - Features of the reference that this build does not implement are
 *    rejected by fb_create with FB_ERR_UNSUPPORTED, never silently ignored.
 */
#ifndef FARGO_B200_H
#define FARGO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define FB_ABI_VERSION 2

#define FB_OK               0
#define FB_ERR_INVALID     -1   /* bad argument or parameter value          */
#define FB_ERR_UNSUPPORTED -2   /* .par feature outside this build          */
#define FB_ERR_CUDA        -3   /* CUDA runtime error                        */
#define FB_ERR_NOMEM       -4   /* device or host allocation failed          */
#define FB_ERR_NAN         -5   /* NaN/Inf found in the gas state            */
#define FB_ERR_NEGATIVE    -6   /* the reference's crash test fired during the
                                   DT (DetectCrash, src/SourceEuler.c:51-69,
                                   545-566): a warning, the DT is complete   */
#define FB_ERR_SUBSTEPS    -7   /* CFL substep count above the cap           */
#define FB_ERR_TIMEOUT     -8   /* a bounded device wait gave up             */
#define FB_ERR_IO          -9   /* file could not be read or written         */
#define FB_ERR_STATE      -10   /* call made in the wrong order              */
#define FB_ERR_NODEVICE   -11   /* no CUDA device visible                    */

#define FB_MAX_PLANETS 16

/* Hot-path parameters.  Field names follow the reference's .par keys
 * (src/var.c:13-202); defaults are the reference's (fb_params_default).
 * String switches are decoded by first letter as src/Interpret.c:165-479
 * does. */
typedef struct fb_params {
  /* grid: NRAD, NSEC, RMIN, RMAX, RADIALSPACING (L/A), PMIN, PMAX */
  int nrad, nsec;
  double rmin, rmax;
  int log_grid;
  double pmin, pmax;
  /* time: DT, NTOT, NINTERM */
  double dt;
  int ntot, ninterm;
  /* disc: SIGMA0, SIGMASLOPE, ASPECTRATIO, FLARINGINDEX */
  double sigma0, sigmaslope, aspectratio, flaringindex;
  /* ALPHAVISCOSITY, VISCOSITY */
  double alphaviscosity, viscosity;
  /* thermodynamics: ADIABATICINDEX, ENERGYEQUATION, VISCOUSHEATING,
     BETACOOLING, BETACOOLINGTIME, BETACOOLINGSLOPE; thermal cooling below */
  double adiabaticindex;
  int energy_equation, viscous_heating, beta_cooling;
  double betacoolingtime, betacoolingslope;
  /* THERMALCOOLING (radiative cooling with Bell & Lin opacities),
     SETCONSTANTOPACITY, IMPOSEDCONSTANTOPACITY, FACTOROPACITIES;
     STELLARIRRADIATION (0 No, 1 Yes: a background temperature
     BACKGROUNDTEMPERATURE r^SLOPEBACKGROUNDTEMPERATURE, 2 L: heating by a
     star of STELLARLUMINOSITY solar luminosities) */
  int thermal_cooling, constant_opacity;
  double imposedconstantopacity, factoropacities;
  int stellar_irradiation;
  double backgroundtemperature, slopebackgroundtemperature, stellarluminosity;
  /* self-gravity: SELFGRAVITY (Yes), SGTHICKNESSSMOOTHING */
  int self_gravity;
  double sgthicknesssmoothing;
  /* planets and frame: THICKNESSSMOOTHING, ROCHESMOOTHING,
     INDIRECTTERMSMOOTHING, MASSTAPER, OMEGAFRAME, INDIRECTTERM,
     DISCARDGASINDIRECTTERM, ALTERNATIVEGASINDIRECTTERM, FORCEDCIRCULAR,
     EXCLUDEHILL, EXCLUDEHILLFACTOR, ECCENTRICITY, RELEASEDATE,
     RELEASERADIUS */
  double thicknesssmoothing, rochesmoothing, indirecttermsmoothing;
  double masstaper, omegaframe;
  int indirect_term, discard_gas_indirect_term, alternative_gas_indirect_term;
  int forced_circular, exclude_hill;
  double excludehillfactor, eccentricity, releasedate, releaseradius;
  /* transport and boundaries: TRANSPORT (FARGO/Standard), INNERBOUNDARY
     (Wall, Open, KNOpen, NonReflecting), WAVEKILLINGZONES, WKZRMIN, WKZRMAX,
     DAMPINGTODYNAMICALTIMERATIO, DAMPTOAXI/DAMPTOINI, ADDFLOORS,
     DENSITYFLOOR, ZEROVRADBC */
  int fast_transport, wall_boundary, evanescent;
  double wkzrmin, wkzrmax, dampingtodynamicaltimeratio;
  int damp_to_axi, damp_to_ini, add_floors;
  double densityfloor;
  int zero_vrad_bc;
  /* INNERBOUNDARY other than WALL (src/Interpret.c:168-175): OPEN (open_inner),
     KNOPEN (open_inner and kn_open: Kley & Nelson's outflow), NONREFLECTING
     (non_reflecting); ACCRETING is refused */
  int open_inner, kn_open, non_reflecting;
  /* MINDT, MAXDT: initial values of the running min/max substep (the
     reference keeps them as .par variables, src/var.c:145-146) */
  double mindt, maxdt;
  /* IMPOSEDDISKDRIFT */
  double imposeddiskdrift;
  /* units: FACTORUNITMASS, FACTORUNITLENGTH, FACTORMMW */
  double factorunitmass, factorunitlength, factormmw;
  /* Lagrangian dust particles: NBPART, SIZEMINPART, SIZEMAXPART,
     SIZEPARTSLOPE, RHOPART, DUSTSLOPE, RMINDUST, RMAXDUST, DUSTFEELDISK,
     DUSTFEELPLANETS, DUSTFEELTURB, DUSTFEEDBACK, DUSTFEELSG, SFTAPPROX,
     INTERPOLATION, WRITEDUSTDENSITY (which makes AlgoGas interpolate the
     gas onto the particles a second time each substep, src/SourceEuler.c:529,
     and so changes the Stokes numbers the next turbulent kick uses) */
  int nbpart;
  double sizeminpart, sizemaxpart, sizepartslope, rhopart, dustslope;
  double rmindust, rmaxdust;
  int dust_feel_disk, dust_feel_planets, dust_feel_turb, dust_feedback, dust_feel_sg;
  int sfta, interpolation; /* interpolation: 0 NGP, 1 CIC, 2 TSC */
  int write_dust_density;
  /* bit mask of .par features that were set but that this build does not
     implement (fb_create refuses a non-zero mask); see fb_unsupported_name */
  unsigned long long unsupported;
  /* PLANETCONFIG and OUTPUTDIR, as written in the .par file */
  char planetconfig[512];
  char outputdir[512];
  /* stochastic turbulent potential of Laughlin et al. (2004) as modified by
     Baruteau & Lin (2010) (src/turb.c:13-135, MHD L): NBTURBMODES modes
     (at most FB_LSA_MAX_MODES), GAMMATURB, LSAMODESPEEDUP, TURBRMIN,
     TURBRMAX, HIGHMCUTOFF (only modes m <= 6), and the cavity profile of
     the forcing amplitude CAVITYRADIUS, CAVITYRATIO, CAVITYWIDTH */
  int mhd_lsa, nbturbmodes, high_m_cutoff;
  double gammaturb, lsamodespeedup, turbrmin, turbrmax;
  double cavityradius, cavityratio, cavitywidth;
  /* thermal diffusion with the energy equation (src/SourceEuler.c:722-762,
     1740-2052): ENTROPYDIFFUSION (explicit, coefficient DIFFUSIVITY) and
     RADIATIVEDIFFUSION, 0 No, 1 E (explicit, flux-limited, Bell & Lin
     opacities of the current state), 2 I (implicit: red-black successive
     over-relaxation, needs an even NSEC) */
  int entropy_diffusion, radiative_diffusion;
  double diffusivity;
  /* FRAME C: a frame corotating with the first planet (OMEGAFRAME is then
     the planet's angular frequency at the start and follows it at every
     substep, src/main.c:228-247, src/SourceEuler.c:476-525); the guiding-
     centre and binary-centre frames (G, B) are refused */
  int corotating;
  /* ADDNOISE: white noise of relative amplitude 1e-3 on the initial density
     (src/Pframeforce.c:317-320), drawn by fb_init_state from the drand48
     stream seeded with its noise_seed (the reference seeds it from the wall
     clock, src/Interpret.c:373-376); TEMPPRESC: relaxation of the energy
     towards its initial profile in SubStep3 (src/SourceEuler.c:1159-1175)
     on the time PRESCTIME0 r^(2+2 FLARINGINDEX) (with VISCOSITY > 0) or
     PRESCTIME0 / Omega */
  int add_noise, temppresc;
  double presctime0;
} fb_params;

#define FB_LSA_MAX_MODES 256

/* Planetary system (src/types.h:96-108).  initial_mass/final_mass are the
   reference's InitialPlanetMass/FinalPlanetMass (src/global.h). */
typedef struct fb_planets {
  int nb;
  double mass[FB_MAX_PLANETS], x[FB_MAX_PLANETS], y[FB_MAX_PLANETS];
  double vx[FB_MAX_PLANETS], vy[FB_MAX_PLANETS], acc[FB_MAX_PLANETS];
  double initial_mass[FB_MAX_PLANETS], final_mass[FB_MAX_PLANETS];
  int feeldisk[FB_MAX_PLANETS], feelothers[FB_MAX_PLANETS], binary[FB_MAX_PLANETS];
} fb_planets;

/* Host view of the state that AlgoGas reads and writes.  Field pointers
   refer to caller-owned arrays of (nrad+1)*nsec doubles; a NULL field is
   skipped by fb_upload / fb_download. */
typedef struct fb_state {
  double *dens, *vrad, *vtheta, *energy;
  double physical_time, physical_time_initial;
  double omega_frame, lost_mass, mindt, maxdt;
  double stardiscbarycenter_x[3], stardiscbarycenter_y[3];
  fb_planets planets;
} fb_state;

/* Axisymmetric profiles the step reads (src/global.h: SigmaMed, SigmaInf,
   EnergyMed, VthetaMed, VradMed, GLOBAL_SoundSpeed), nrad doubles each. */
typedef struct fb_profiles {
  double *sigma_med, *sigma_inf, *energy_med, *vtheta_med, *vrad_med;
  double *global_soundspeed;
} fb_profiles;

/* What one fb_algogas call did.
   Crash bookkeeping follows AlgoGas (src/SourceEuler.c:545-566): at every
   substep the state is tested for negative values before the gas update, and
   the substep "crashes" when the energy is negative somewhere (the density
   test runs too, but its result is overwritten by the energy test's, so an
   isothermal run never crashes).  The first crash's time is timeCRASH and its
   state (density, vrad, vtheta, energy of rings 0..nrad-1) is kept on the
   device for fb_download_crash, the reference's *999.dat dumps.  Like the
   reference, the step carries on after a crash: fb_algogas completes the DT
   and returns FB_ERR_NEGATIVE (status too) when any of its substeps crashed. */
typedef struct fb_step_report {
  int substeps;          /* CFL substeps taken in this DT                 */
  int status;            /* FB_OK or the first error seen                 */
  double physical_time;  /* PhysicalTime after the DT                      */
  double mindt, maxdt;   /* MINDT / MAXDT (src/SourceEuler.c:457-460)     */
  double lost_mass;      /* LostMass (src/TransportEuler.c:137)            */
  double gpu_ms;         /* device time of the DT (CUDA events)            */
  int crashes;           /* AlreadyCrashed: crashed substeps so far (since
                            fb_create), src/SourceEuler.c:563           */
  int crash_substeps;    /* crashed substeps of this DT (the 'c' marks of
                            src/SourceEuler.c:564)                       */
  int neg_density_substeps; /* substeps of this DT that began with a negative
                            density somewhere (not a crash for AlgoGas)  */
  double crash_time;     /* timeCRASH: PhysicalTime of the first crash
                            (src/SourceEuler.c:551); 0 if none           */
  double disk_on_primary[2]; /* DiskOnPrimaryAcceleration (x, y) of the last
                            substep (src/SourceEuler.c:482), which the
                            reference's planet logs read after AlgoGas    */
  double disk_on_primary_alt[2]; /* DiskOnPrimaryAcceleration_alt (x, y), the
                            barycentre's finite-difference version
                            (src/SideEuler.c:91-112), for the
                            compindirectterm.dat output (src/Output.c)   */
} fb_step_report;

/* Lagrangian dust particles (src/types.h:114-146, the fields the step
   carries between DTs).  Arrays are caller-owned, n doubles each.  rng_x
   is the 48-bit drand48 state after every draw made so far; kicks counts
   the turbulent-kick calls made so far by each of the two Gaussian
   generators of src/DustUpdate.c:438-485, and carry holds their cached
   second deviates (radial, azimuthal) when kicks is odd. */
typedef struct fb_dust_state {
  int n;
  double *r, *th, *vr, *vth, *l, *size, *stokes;
  unsigned long long rng_x;
  long long kicks;
  double carry[2];
  double particles_mass;   /* Particles_Mass (main.c:190-224) */
} fb_dust_state;

/* Download masks */
#define FB_F_DENS    0x01u
#define FB_F_VRAD    0x02u
#define FB_F_VTHETA  0x04u
#define FB_F_ENERGY  0x08u
#define FB_F_ALL     0x0Fu

typedef struct fb_ctx fb_ctx;

/* ---- parameters (host only, no GPU needed) --------------------------- */
/* Defaults of src/var.c:13-202 and src/Interpret.c:23-50. */
int fb_params_default(fb_params *p);
/* Reads a .par file with the rules of ReadVariables (src/Interpret.c:82-480):
   case-insensitive keys, '#' comments, separators "\t :=>_".  Unknown keys
   are ignored like the reference does (it warns). */
int fb_params_read_par(fb_params *p, const char *path);
/* Name of the first unsupported feature in p->unsupported, or "" */
const char *fb_unsupported_name(const fb_params *p);

/* ---- initial conditions (host only) ------------------------------------ */
/* Reads the planet .cfg file (InitPlanetarySystem, src/Psys.c:96-203). */
int fb_planets_read_cfg(const fb_params *p, const char *path, fb_planets *out);
/* Fills state and profiles exactly as the reference's main.c:145-291 does
   for the supported features: FillPolar1DArrays, InitGasDensity (+ optional
   seeded white noise of relative amplitude noise_amp, drawn with the POSIX
   drand48 stream seeded by noise_seed, in the reference's loop order),
   InitGasEnergy, InitEuler/InitGasVelocities.  With self-gravity the
   initial SG acceleration is needed, which is computed on the GPU of ctx;
   pass ctx = NULL otherwise.  Field arrays must be allocated by the caller. */
int fb_init_state(const fb_params *p, fb_ctx *ctx, double noise_amp,
                  long noise_seed, fb_state *st, fb_profiles *prof);

/* Draws the initial particles exactly as InitDustSystem does
   (src/Dsys.c:128-262): sizes, then radii, then azimuths from the POSIX
   drand48 stream seeded with `seed`; Keplerian azimuthal velocities (with
   the self-gravity correction when ctx holds self-gravity).  Arrays of
   st->n = p->nbpart doubles must be allocated by the caller. */
int fb_init_dust(const fb_params *p, fb_ctx *ctx, long seed, fb_dust_state *st);

/* ---- device context ------------------------------------------------------ */
/* Selects the CUDA device used by contexts created afterwards on this host
   thread (cudaSetDevice of the library's runtime). */
int fb_select_device(int device);
/* radii: optional nrad+1 interface radii (the reference's Radii array,
   src/SourceEuler.c:88-104); NULL computes them from rmin/rmax/log_grid. */
int fb_create(const fb_params *p, const double *radii, fb_ctx **out);
int fb_destroy(fb_ctx *ctx);
int fb_upload(fb_ctx *ctx, const fb_state *st, const fb_profiles *prof);
/* One DT of AlgoGas (src/SourceEuler.c:326-719) on device-resident state. */
int fb_algogas(fb_ctx *ctx, fb_step_report *rep);
int fb_download(fb_ctx *ctx, fb_state *st, unsigned mask);
/* Particles (NBPART > 0): upload once after fb_upload (computes the
   particles' gas values and Stokes numbers as the reference's first
   interpolation call, src/main.c:287), download when writing outputs. */
int fb_dust_upload(fb_ctx *ctx, const fb_dust_state *st);
int fb_dust_download(fb_ctx *ctx, fb_dust_state *st);
/* Turbulent potential (MHD L, ApplyLSAOnPotential, src/turb.c:13-135): the
   modes are drawn on the device from the POSIX drand48 stream, the
   reference's global one (seeded at src/Interpret.c:404-407, then used by
   whatever draws before the time loop).  The stream's 48-bit state is read
   (set = 0) or written (set = 1) here; a context starts with srand48(0)'s.
   fb_rand48_state gives srand48(seed)'s state advanced by `draws` draws
   (with noise, fb_init_state draws nrad*nsec numbers after seeding).
   Every mode is redrawn at the first substep after fb_create, as the
   reference's zeroed mode lifetimes make it do at the start of a run. */
int fb_lsa_stream(fb_ctx *ctx, unsigned long long *x, int set);
unsigned long long fb_rand48_state(long seed, long long draws);
/* The state at the first crash (see fb_step_report), nrad*nsec doubles per
   non-NULL field of st (density, vrad, vtheta, energy; ring nrad untouched):
   what the reference writes as gasdens999.dat, gasvrad999.dat,
   gasvtheta999.dat and gasenergy999.dat (src/SourceEuler.c:549-561).
   FB_ERR_STATE if no crash happened. */
int fb_download_crash(fb_ctx *ctx, fb_state *st, double *crash_time);
/* Derived output fields at the current state (reference layout, (nrad+1)*nsec):
   which = 0 Temperature (src/SourceEuler.c:2440), 1 Potential, 2 Pressure,
   3 SoundSpeed, 4 DivergenceVelocity, 5 ViscHeat, 6 SG radial acceleration
   (SG_Accr, src/sgacc.c:152-161), 7 SG azimuthal acceleration (SG_Acct). */
int fb_download_derived(fb_ctx *ctx, int which, double *out);
/* Rings [ring0, ring0+nrings) of the self-gravity accelerations last
   computed (by the step, or by fb_stage(.., FB_STAGE_SELFGRAV, ..)): SG_Accr
   and SG_Acct of src/sgacc.c:152-161, into accr / acct (either may be NULL)
   at their own offsets of (nrad+1)*nsec arrays.  The reference's planet log
   UpdateLogSG (src/Force.c:331) reads only the rings next to each planet. */
int fb_download_sgacc(fb_ctx *ctx, int ring0, int nrings, double *accr, double *acct);
/* Diagnostics on the device state: GasTotalMass (src/SideEuler.c:15) and
   GasMomentum (src/SideEuler.c:114). */
int fb_diagnostics(fb_ctx *ctx, double *mass, double *momentum);
/* ComputeForce (src/Force.c:77-253) of the disc's current density on a body
   at (x, y) with smoothing length rsmoothing and mass `mass`, with the Hill
   cut of EXCLUDEHILLFACTOR: out[8] = fx_inner, fx_ex_inner, fx_outer,
   fx_ex_outer, fy_inner, fy_ex_inner, fy_outer, fy_ex_outer (the Force
   fields).  Summed per ring on the device, then over the rings in ring
   order (about 1e-16 relative from the reference's single sequential sum).
   It serves the per-DT planet logs (UpdateLog, src/Force.c:266-328) without
   a download of the density. */
int fb_planet_force(fb_ctx *ctx, double x, double y, double rsmoothing, double mass, double *out);
/* ---- launch shapes (no counterpart in the reference) ---------------------
   CTA width of the per-cell kernels (32..256, multiple of 32), cells per
   thread of the azimuthal transport (1..4), columns (32/64/128) and rings
   per CTA of the radial transport.  0 in fb_set_tuning means automatic;
   fb_get_tuning reports the values in effect.  fb_tune times the candidates
   on the context's own disc, `substeps` substeps each from a saved state
   that it restores (the disc does not advance), keeps the fastest and
   reports the summed ms per substep of the tuned stages. */
typedef struct fb_tuning {
  int cell_block, azi_cells_per_thread, rad_columns, rad_rings;
  int azi_variant;  /* 0 automatic, 1 narrow (NQ+3 shared rings), 2 wide (2 NQ+1 rings),
                       3 packed (12 rings, 13 with energy; a cell's quantities side by side),
                       4 register (E = 2..4 contiguous cells per thread, quantities in
                       registers; nsec = E T with T a multiple of 32), 5 staged (the
                       register variant in a persistent kernel whose rings arrive and
                       leave by bulk asynchronous copies, one ring ahead), 6 tile (the
                       register variant's arithmetic with one warp per tile of
                       32 E - 9 cells and no barrier; E = 2..4; four CTAs of four
                       warps per SM), 7 (the tile variant with up to 168
                       registers a thread: three CTAs per SM), 8 (the tile
                       variant at five CTAs per SM, 96 registers) */
} fb_tuning;
int fb_get_tuning(const fb_ctx *ctx, fb_tuning *t);
int fb_set_tuning(fb_ctx *ctx, const fb_tuning *t);
int fb_tune(fb_ctx *ctx, int substeps, fb_tuning *best, double *ms_per_substep);

/* ---- batches of discs (no counterpart in the reference) ----------------- */
/* Many discs -- contexts of any grid size and parameters on the current
   device, each uploaded -- advanced one DT each by one graph launch, their
   substep loops running side by side on the GPU.  A context may belong to
   one batch at a time and keeps working on its own with fb_algogas. */
typedef struct fb_batch fb_batch;
int fb_batch_create(fb_ctx *const *ctxs, int n, fb_batch **out);
/* One DT of every disc; reps (n entries, may be NULL) as fb_algogas reports
   them, gpu_ms being the whole batch's device time.  Returns the first
   non-zero disc status. */
int fb_batch_algogas(fb_batch *b, fb_step_report *reps);
int fb_batch_destroy(fb_batch *b);

/* ---- learned coarse-grid closure (no counterpart in the reference) -------
   A 4-layer periodic-in-azimuth CNN (3x3 convolutions, 32 channels, GELU;
   BF16 weights and activations, FP32 accumulation on the tensor cores) that
   reads a coarse disc and returns two face fluxes of mass per cell (in units
   of scale x the disc's initial density at the face), applied as flux
   differences; the corrected mass carries its upwind angular momentum, so
   mass and angular momentum change only by round-off.  The coarse grid's
   nsec must be a multiple of 64; isothermal discs.  Training samples live
   on the device: for sample s, fb_closure_record(.., s, 0) stores the input
   features (and the initial density profile) of the coarse disc, (.., s, 1)
   subtracts its conservative variables after the plain method's DT, (.., s,
   2) adds those of the coarse-grained fine disc one DT later (the target). */
typedef struct fb_closure fb_closure;
int fb_closure_create(const fb_ctx *coarse, int capacity, int batch, unsigned long long seed, fb_closure **out);
int fb_closure_destroy(fb_closure *c);
int fb_closure_num_params(const fb_closure *c, int *nweights, int *nbiases);
/* get = 1 copies FP32 weights ([out][tap][in] per layer) and biases out,
   get = 0 sets them */
int fb_closure_params(fb_closure *c, float *w, float *b, int get);
/* 3 output scales and 3 loss weights (entry 0: mass; 1, 2 unused), get or set */
int fb_closure_scales(fb_closure *c, double *scale, double *wq, int get);
/* scale and weight from the first `count` samples:
   rms(target * Surf / Sigma0), 1/mean(target^2) */
int fb_closure_autoscale(fb_closure *c, int count);
int fb_closure_record(fb_closure *c, fb_ctx *coarse, int slot, int what);
/* host-provided sample: x = nrad*nsec*16 feature floats (rounded to BF16),
   y = 3*nrad*nsec targets (mass, angular and radial momentum; the loss
   uses the mass), sig = nrad initial densities of the sample's disc */
int fb_closure_set_sample(fb_closure *c, int slot, const float *x, const float *y, const float *sig);
/* loss and gradients (same layout as fb_closure_params) of samples
   [first, first+nb), no update; gw/gb may be NULL */
int fb_closure_loss_grad(fb_closure *c, int first, int nb, double *loss, float *gw, float *gb);
/* `iters` Adam steps on random minibatches of nb samples of [first,
   first+count); loss_out[iters] optional */
int fb_closure_train(fb_closure *c, int first, int count, int nb, int iters, double lr, unsigned long long seed,
                     double *loss_out);
/* network output (nrad*nsec*16 floats, channels 0, 1 = the mass fluxes)
   for sample slot, or for the coarse disc's state when slot < 0 */
int fb_closure_infer(fb_closure *c, const fb_ctx *coarse, int slot, float *out);
/* one correction of the coarse disc's state (density and vtheta), in
   place; each face flux is saturated at 3 output scales (3 tanh(F/3), a
   conservative map) and multiplied by the gain (default 1) */
int fb_closure_apply(fb_closure *c, fb_ctx *coarse);
int fb_closure_set_gain(fb_closure *c, double gain);
/* coarse disc := coarse-graining of a fine disc on the same radii whose
   grid is an integer multiple in both directions (isothermal) */
int fb_downsample(const fb_ctx *fine, fb_ctx *coarse);

/* No counterpart in the reference (it has no vortensity routine): the
   vortensity xi = omega_z / Sigma at the cell corners (R_inf[i], phi_inf[j]),
   i = 1..nrad-1, with omega_z = [d(R vtheta)/dR - d(vrad)/dphi] / R_inf
   + 2 OmegaFrame from centred differences of the staggered velocities and
   Sigma the mean of the four cells around the corner (ring 0 and ring nrad
   are 0); and the azimuthal means of Sigma (per ring) and of xi (per
   interface ring).  Any output may be NULL: field (nrad+1)*nsec doubles,
   sigma_mean and vort_mean nrad doubles. */
int fb_vortensity(fb_ctx *ctx, double *field, double *sigma_mean, double *vort_mean);
const char *fb_strerror(int code);
const char *fb_last_error(const fb_ctx *ctx);

/* ---- single stages (parity tests and profiling) ------------------------ */
#define FB_STAGE_TRANSPORT  1  /* Transport (src/TransportEuler.c:65)       */
#define FB_STAGE_VISCOSITY  2  /* ComputeViscousTerms + UpdateVelocitiesWithViscosity
                                  on (vrad, vtheta, dens) (src/Viscosity.c:159-378) */
#define FB_STAGE_BOUNDARY   3  /* ApplyBoundaryCondition (src/SideEuler.c:1102): walls,
                                  sub-Keplerian edges, open and non-reflecting edges */
#define FB_STAGE_DAMPING    4  /* EvanescentBoundary (src/SideEuler.c:796)  */
#define FB_STAGE_SELFGRAV   5  /* compute_sgacc only: fills SG accelerations */
int fb_stage(fb_ctx *ctx, int stage, double dt);

/* ---- allocation-free transport -------------------------------------------- */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc:
   host codes embedded in a GPU application that owns the whole device-memory
   budget, or that call from regions where an allocation (which may also
   synchronize the device) is not acceptable.  Runs the same kernels as
   fb_stage(ctx, FB_STAGE_TRANSPORT, dt) (Transport, src/TransportEuler.c:65)
   without a context and without allocating anything: the inter-pass scratch
   is a fixed file-scope device array of at most FB_NOALLOC_MAX_CELLS cells
   (about 7.4 MB), held on a GPU from the first call there until exit.
   dens, vrad, vtheta, energy are DEVICE pointers to (nrad+1)*nsec doubles in
   the PolarGrid layout, updated in place (energy only with the energy
   equation); stream is a cudaStream_t (NULL: default stream); lost_mass, if
   not NULL, receives the ring-0 outflow of this call (the stream is then
   synchronized).  Grids with (nrad+1)*nsec > FB_NOALLOC_MAX_CELLS, nrad >
   4096 or nsec > 3072 are refused with FB_ERR_INVALID.  The first call on a
   device sets up the device addresses and loads every kernel a call can
   launch: it is the only call that may make the CUDA driver allocate (module
   loading); later calls allocate nothing.  Every call copies the grid tables
   from host memory and synchronizes the stream, so no call may be made while
   its stream is being captured into a CUDA graph.  All calls share the
   scratch, so calls that overlap on the GPU race.  The reason for a failure
   is in fb_noalloc_last_error(). */
#define FB_NOALLOC_MAX_CELLS 131072
int fb_transport_noalloc(const fb_params *p, double *dens, double *vrad, double *vtheta,
                         double *energy, double dt, void *stream, double *lost_mass);
const char *fb_noalloc_last_error(void);

/* ---- profiling ----------------------------------------------------------- */
/* Number of kernel launches this context has issued. */
long long fb_kernel_launches(const fb_ctx *ctx);
/* enable = 1: record CUDA events between the stages of every substep and
   accumulate each stage's device time (adds event records to the stream,
   for profiling runs); enable = 0 stops.  Resets the accumulators. */
int fb_profile(fb_ctx *ctx, int enable);
/* Stage idx (0 .. n-1) of the profile: its name, accumulated device ms and
   number of launches; returns the number of stages, or a negative code. */
int fb_profile_read(const fb_ctx *ctx, int idx, const char **name, double *ms, long long *launches);

/* Build information: "sm_100a fp64 ..." */
const char *fb_build_info(void);
/* sizeof of the ABI structs (0 fb_params, 1 fb_planets, 2 fb_state,
   3 fb_profiles, 4 fb_step_report, 5 fb_dust_state, 6 fb_tuning), for
   bindings to check their layout. */
int fb_struct_size(int which);

#ifdef __cplusplus
}
#endif
#endif /* FARGO_B200_H */
