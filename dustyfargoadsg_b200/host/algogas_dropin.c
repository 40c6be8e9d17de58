/* algogas_dropin.c -- AlgoGas for the reference's own driver, running on the
 * GPU through libfargo_b200.so.
 *
 * A maintainer links this file into the reference build and either names
 * the function AlgoGas (removing SourceEuler.c's), or keeps both and links
 * with -Wl,--wrap=AlgoGas and a one-line __wrap_AlgoGas that calls
 * fb_dropin_AlgoGas.  The signature is the reference's
 * (src/SourceEuler.c:326-331, src/proto.h:82).  It is compiled against the
 * reference's headers (mp.h and the generated param.h / global_ex.h), so the
 * .par globals are read directly.
 *
 * First call: translate the globals into fb_params, create the context with
 * the reference's own Radii, upload the fields, profiles and planets.  Every
 * call: one DT on the GPU, then the host PolarGrids, planets, particles, the
 * drand48 stream and the scalar globals (PhysicalTime, LostMass, MINDT,
 * MAXDT, stardiscbarycenter) are refreshed so that the reference's
 * SendOutput, planet and particle logs and -a monitor see the state they
 * expect.  A crash (the reference's negative-energy test) is reported as the
 * reference does: "Crash!" and the *999.dat dumps once, a 'c' per crashed
 * substep, and the run goes on.  Errors print a message and call prs_exit(1),
 * the reference's own way of stopping (src/LowTasks.c:32).
 */
#include "mp.h"
#include "fargo_b200.h"
#include "fb_internal.h"

extern real LostMass;
extern boolean SelfGravity, SGZeroMode, EnergyEquation, ViscousHeating, BetaCooling;
extern boolean FastTransport, WallBoundary, Evanescent, DampToAxi, DampToIni, DampToViscous;
extern boolean AddFloors, ImposeZeroRadialVelocityBC, Indirect_Term, Discard_GasIndirect_term;
extern boolean Alternative_Gas_Indirect_Term, ForcedCircular, ForcedInnerCircular, ExcludeHill;
extern boolean OpenInner, NonReflecting, AccBoundary, OuterSourceMass, Corotating, DustFluid;
extern boolean AdvecteLabel, ZMPlus, MHDLSA, EntropyDiffusion, RadiativeDiffusion, ThermalCooling;
extern boolean TempPresc, AddMass, DiscEvaporation, PhotoEvaporation, CavityTorque, ComputeCPDMass;
extern boolean BM08, DustFeedback, Write_Temperature, Write_Potential;
extern boolean DustFeelDisk, DustFeelPlanets, DustFeelTurb, DustFeelSG, DustFeelSGZeroMode;
extern boolean ShortFrictionTimeApproximation, TSCInterpolation, Write_DustDensity, ZZIntegrator;
extern boolean DustGrowth, RemoveDustFromPlanetsHillRadius, NoTimestepConstraintByParticles, SoftWriting;
extern boolean CompareSGAndSummationTorques, KNOpen, SetConstantOpacity, StellarIrradiation, ImposedStellarLuminosity;
extern boolean HighMCutoff, ImplicitRadiativeDiffusion, GuidingCenter, BinaryCenter, CorotateWithOuterPlanet;
extern Pair DiskOnPrimaryAcceleration, DiskOnPrimaryAcceleration_alt;

static fb_ctx *g_ctx = NULL;
static int g_crashes = 0;  /* AlreadyCrashed as last reported */
static long g_substeps = 0; /* CFL substeps of all DTs so far */
/* the host state the last DT left behind: downloaded on demand */
static int g_host_stale = 0, g_sync_always = 0;
static PolarGrid *g_rho, *g_vrad, *g_vtheta, *g_energy;
static DustSystem *g_dsys;
static PlanetarySystem *g_sys;

static void dropin_fail(const char *what, int rc)
{
  mastererr("libfargo_b200: %s failed: %s (%s)\n", what, fb_strerror(rc), fb_last_error(g_ctx));
  prs_exit(1);
}

static void params_from_globals(fb_params *p)
{
  fb_params_default(p);
  p->nrad = GLOBALNRAD;
  p->nsec = NSEC;
  p->rmin = RMIN;
  p->rmax = RMAX;
  p->log_grid = LogGrid;
  p->pmin = PMIN;
  p->pmax = PMAX;
  p->dt = DT;
  p->ntot = NTOT;
  p->ninterm = NINTERM;
  p->sigma0 = SIGMA0;
  p->sigmaslope = SIGMASLOPE;
  p->aspectratio = ASPECTRATIO;
  p->flaringindex = FLARINGINDEX;
  p->alphaviscosity = ALPHAVISCOSITY;
  p->viscosity = VISCOSITY;
  p->adiabaticindex = ADIABATICINDEX;
  p->energy_equation = EnergyEquation;
  p->viscous_heating = ViscousHeating;
  p->beta_cooling = BetaCooling;
  p->betacoolingtime = BETACOOLINGTIME;
  p->betacoolingslope = BETACOOLINGSLOPE;
  p->self_gravity = SelfGravity;
  p->sgthicknesssmoothing = SGTHICKNESSSMOOTHING;
  p->thicknesssmoothing = THICKNESSSMOOTHING;
  p->rochesmoothing = ROCHESMOOTHING;
  p->indirecttermsmoothing = INDIRECTTERMSMOOTHING;
  p->masstaper = MASSTAPER;
  p->omegaframe = OMEGAFRAME;
  p->indirect_term = Indirect_Term;
  p->discard_gas_indirect_term = Discard_GasIndirect_term;
  p->alternative_gas_indirect_term = Alternative_Gas_Indirect_Term;
  p->forced_circular = ForcedCircular;
  p->exclude_hill = ExcludeHill;
  p->excludehillfactor = EXCLUDEHILLFACTOR;
  p->eccentricity = ECCENTRICITY;
  p->releasedate = RELEASEDATE;
  p->releaseradius = RELEASERADIUS;
  p->fast_transport = FastTransport;
  p->wall_boundary = WallBoundary;
  p->evanescent = Evanescent;
  p->wkzrmin = WKZRMIN;
  p->wkzrmax = WKZRMAX;
  p->dampingtodynamicaltimeratio = DAMPINGTODYNAMICALTIMERATIO;
  p->damp_to_axi = DampToAxi;
  p->damp_to_ini = DampToIni;
  p->add_floors = AddFloors;
  p->densityfloor = floordens;
  p->zero_vrad_bc = ImposeZeroRadialVelocityBC;
  p->mindt = MINDT;
  p->maxdt = MAXDT;
  p->imposeddiskdrift = IMPOSEDDISKDRIFT;
  p->factorunitmass = FACTORUNITMASS;
  p->factorunitlength = FACTORUNITLENGTH;
  p->factormmw = FACTORMMW;
  p->nbpart = NBPART;
  /* features the GPU build does not implement are refused by fb_create */
  p->open_inner = OpenInner;
  p->kn_open = KNOpen;
  p->non_reflecting = NonReflecting;
  if (AccBoundary) p->unsupported |= FB_U_BOUNDARY;
  if (OuterSourceMass) p->unsupported |= FB_U_OUTERSOURCE;
  if (DampToViscous) p->unsupported |= FB_U_DAMPTOVISCOUS;
  if (AddMass) p->unsupported |= FB_U_ADDMASS;
  if (DiscEvaporation) p->unsupported |= FB_U_EVAPORATION;
  if (PhotoEvaporation) p->unsupported |= FB_U_PHOTOEVAP;
  if (SelfGravity && SGZeroMode) p->unsupported |= FB_U_SGZEROMODE;
  if (ZMPlus) p->unsupported |= FB_U_ZMPLUS;
  /* the turbulent potential (src/turb.c); it shares the drand48 stream
     with the particles, so the two together are refused */
  p->mhd_lsa = MHDLSA;
  p->nbturbmodes = NBTURBMODES;
  p->high_m_cutoff = HighMCutoff;
  p->gammaturb = GAMMATURB;
  p->lsamodespeedup = LSAMODESPEEDUP;
  p->turbrmin = TURBRMIN;
  p->turbrmax = TURBRMAX;
  p->cavityradius = CAVITYRADIUS;
  p->cavityratio = CAVITYRATIO;
  p->cavitywidth = CAVITYWIDTH;
  if (MHDLSA && (NBPART != 0 || NBTURBMODES < 0 || NBTURBMODES > FB_LSA_MAX_MODES)) p->unsupported |= FB_U_MHDLSA;
  p->entropy_diffusion = EntropyDiffusion;
  p->radiative_diffusion = RadiativeDiffusion ? (ImplicitRadiativeDiffusion ? 2 : 1) : 0;
  p->diffusivity = DIFFUSIVITY;
  if (p->radiative_diffusion == 2 && (NSEC % 2) != 0) p->unsupported |= FB_U_THERMALDIFF;
  p->thermal_cooling = ThermalCooling;
  p->constant_opacity = SetConstantOpacity;
  p->imposedconstantopacity = IMPOSEDCONSTANTOPACITY;
  p->factoropacities = FACTOROPACITIES;
  p->stellar_irradiation = StellarIrradiation ? (ImposedStellarLuminosity ? 2 : 1) : 0;
  p->backgroundtemperature = BACKGROUNDTEMPERATURE;
  p->slopebackgroundtemperature = SLOPEBACKGROUNDTEMPERATURE;
  p->stellarluminosity = STELLARLUMINOSITY;
  p->temppresc = TempPresc;
  p->presctime0 = PRESCTIME0;
  p->corotating = Corotating;
  if (GuidingCenter || BinaryCenter || CorotateWithOuterPlanet || (Corotating && NBPART != 0))
    p->unsupported |= FB_U_COROTATING;
  if (BM08) p->unsupported |= FB_U_BM08;
  if (ComputeCPDMass) p->unsupported |= FB_U_CPDMASS;
  if (AdvecteLabel) p->unsupported |= FB_U_LABEL;
  if (CavityTorque || CentrifugalBalance) p->unsupported |= FB_U_CENTRIFUGAL;
  if (DustFluid) p->unsupported |= FB_U_DUSTFLUID;
  if (ForcedInnerCircular) p->unsupported |= FB_U_FORCEDINNER;
  if (CAVITYRADIUS != 0.0 || CAVITYRATIO != 1.0) p->unsupported |= FB_U_CAVITY;
  if (TRANSITIONRADIUS != 0.0 || TRANSITIONRATIO != 1.0) p->unsupported |= FB_U_TRANSITION;
  if (LAMBDADOUBLING != 0.0) p->unsupported |= FB_U_LAMBDADOUBLING;
  if (RELEASEDATE != 0.0) p->unsupported |= FB_U_RELEASE;
  /* Lagrangian particles (Dsys.c, DustUpdate.c) */
  p->sizeminpart = SIZEMINPART;
  p->sizemaxpart = SIZEMAXPART;
  p->sizepartslope = SIZEPARTSLOPE;
  p->rhopart = RHOPART;
  p->dustslope = DUSTSLOPE;
  p->rmindust = RMINDUST;
  p->rmaxdust = RMAXDUST;
  p->dust_feel_disk = DustFeelDisk;
  p->dust_feel_planets = DustFeelPlanets;
  p->dust_feel_turb = DustFeelTurb;
  p->dust_feedback = DustFeedback;
  p->dust_feel_sg = DustFeelSG;
  p->sfta = ShortFrictionTimeApproximation;
  p->interpolation = TSCInterpolation ? 2 : 0;
  p->write_dust_density = Write_DustDensity;
  if (NBPART != 0) {
    if (ZZIntegrator) p->unsupported |= FB_U_ZZINTEGRATOR;
    if (DustGrowth) p->unsupported |= FB_U_DUSTGROWTH;
    if (RemoveDustFromPlanetsHillRadius) p->unsupported |= FB_U_HILLREMOVAL;
    if (!TSCInterpolation) p->unsupported |= FB_U_INTERPOLATION;
    if (DustFeelSGZeroMode) p->unsupported |= FB_U_DUSTSGZERO;
    if (!NoTimestepConstraintByParticles) p->unsupported |= FB_U_DUSTTIMESTEP;
    if (SelfGravity && SoftWriting) p->unsupported |= FB_U_SOFTWRITING;
  }
}

/* The libc drand48 state (X = x[2]:x[1]:x[0]) read and written through
   seed48, which also resets the multiplier and increment to the defaults
   that drand48 uses anyway. */
static unsigned long long rand48_get(void)
{
  unsigned short probe[3] = {0, 0, 0}, keep[3];
  unsigned short *old = seed48(probe);
  keep[0] = old[0];
  keep[1] = old[1];
  keep[2] = old[2];
  seed48(keep);
  return (unsigned long long)keep[0] | ((unsigned long long)keep[1] << 16) | ((unsigned long long)keep[2] << 32);
}

static void rand48_set(unsigned long long x)
{
  unsigned short s[3];
  s[0] = (unsigned short)(x & 0xFFFFu);
  s[1] = (unsigned short)((x >> 16) & 0xFFFFu);
  s[2] = (unsigned short)((x >> 32) & 0xFFFFu);
  seed48(s);
}

static void dust_views(fb_dust_state *d, DustSystem *dsys)
{
  memset(d, 0, sizeof *d);
  d->n = NBPART;
  d->r = dsys->r;
  d->th = dsys->th;
  d->vr = dsys->vr;
  d->vth = dsys->vth;
  d->l = dsys->l;
  d->size = dsys->dustsize;
  d->stokes = dsys->stokesnb;
}

static void state_views(fb_state *st, PolarGrid *Rho, PolarGrid *Vrad, PolarGrid *Vtheta,
                        PolarGrid *Energy)
{
  memset(st, 0, sizeof *st);
  st->dens = Rho->Field;
  st->vrad = Vrad->Field;
  st->vtheta = Vtheta->Field;
  st->energy = Energy->Field;
}

/* The reference's reaction to its first crash (SourceEuler.c:549-561):
   "Crash! at time ..." and the state of that substep written as
   gas{dens,vrad,vtheta,energy}999.dat by its own WriteDiskPolar, here from
   the copy the GPU kept (fb_download_crash). */
static void write_crash_dumps(PolarGrid *Rho, PolarGrid *Vrad, PolarGrid *Vtheta, PolarGrid *Energy)
{
  PolarGrid *g[4];
  double *buf[4];
  real *keep;
  fb_state cs;
  double t = 0.0;
  const size_t n = (size_t)NRAD * NSEC;
  int q, rc;
  g[0] = Rho; g[1] = Vrad; g[2] = Vtheta; g[3] = Energy;
  for (q = 0; q < 4; q++) {
    buf[q] = (double *)malloc(n * sizeof(double));
    if (!buf[q]) dropin_fail("crash dump buffer", FB_ERR_NOMEM);
  }
  memset(&cs, 0, sizeof cs);
  cs.dens = buf[0];
  cs.vrad = buf[1];
  cs.vtheta = buf[2];
  cs.energy = buf[3];
  rc = fb_download_crash(g_ctx, &cs, &t);
  if (rc) dropin_fail("fb_download_crash", rc);
  fprintf(stdout, "\nCrash! at time %.12g\n", t);
  for (q = 0; q < 4; q++) {
    keep = g[q]->Field;
    g[q]->Field = buf[q];
    WriteDiskPolar(g[q], 999);
    g[q]->Field = keep;
    free(buf[q]);
  }
}

long fb_dropin_substeps(void) { return g_substeps; }

/* Brings the fields the last DT left on the GPU (and the particles with the
   position of the drand48 stream) back into the reference's host arrays. */
void fb_dropin_sync_host(void)
{
  fb_state st;
  fb_dust_state dst;
  int rc;
  if (!g_ctx || !g_host_stale) return;
  state_views(&st, g_rho, g_vrad, g_vtheta, g_energy);
  rc = fb_download(g_ctx, &st, FB_F_ALL);
  if (rc) dropin_fail("fb_download", rc);
  if (EnergyEquation || Write_Temperature) {
    rc = fb_download_derived(g_ctx, 0, Temperature->Field);
    if (rc) dropin_fail("fb_download_derived", rc);
  }
  if (Write_Potential) {
    rc = fb_download_derived(g_ctx, 1, Potential->Field);
    if (rc) dropin_fail("fb_download_derived", rc);
  }
  if (NBPART != 0) {
    dust_views(&dst, g_dsys);
    rc = fb_dust_download(g_ctx, &dst);
    if (rc) dropin_fail("fb_dust_download", rc);
    rand48_set(dst.rng_x);
  }
  g_host_stale = 0;
}
#define sync_host fb_dropin_sync_host

void fb_dropin_AlgoGas(Force *force, PolarGrid *Rho, PolarGrid *Vrad, PolarGrid *Vtheta,
                       PolarGrid *Energy, PolarGrid *Label, PolarGrid *DRho,
                       PolarGrid *dustpcdens, PolarGrid *DVrad, PolarGrid *DVtheta,
                       PlanetarySystem *sys, DustSystem *dsys)
{
  fb_state st;
  fb_step_report rep;
  int rc, k;
  fb_dust_state dst;
  (void)force; (void)Label; (void)DRho; (void)dustpcdens; (void)DVrad; (void)DVtheta;
  state_views(&st, Rho, Vrad, Vtheta, Energy);
  g_sys = sys;
  if (!g_ctx) {
    const char *sync = getenv("FB_DROPIN_SYNC");
    g_sync_always = (sync && atoi(sync) != 0);
    fb_params p;
    fb_profiles prof;
    params_from_globals(&p);
    if (sys->nb > FB_MAX_PLANETS) dropin_fail("planet count", FB_ERR_UNSUPPORTED);
    rc = fb_create(&p, Radii, &g_ctx);
    if (rc) dropin_fail("fb_create", rc);
    st.physical_time = PhysicalTime;
    st.physical_time_initial = PhysicalTimeInitial;
    st.omega_frame = OmegaFrame;
    st.lost_mass = LostMass;
    st.mindt = MINDT;
    st.maxdt = MAXDT;
    for (k = 0; k < 3; k++) {
      st.stardiscbarycenter_x[k] = stardiscbarycenter_x[k];
      st.stardiscbarycenter_y[k] = stardiscbarycenter_y[k];
    }
    st.planets.nb = sys->nb;
    for (k = 0; k < sys->nb; k++) {
      st.planets.mass[k] = sys->mass[k];
      st.planets.x[k] = sys->x[k];
      st.planets.y[k] = sys->y[k];
      st.planets.vx[k] = sys->vx[k];
      st.planets.vy[k] = sys->vy[k];
      st.planets.acc[k] = sys->acc[k];
      st.planets.initial_mass[k] = InitialPlanetMass[k];
      st.planets.final_mass[k] = FinalPlanetMass[k];
      st.planets.feeldisk[k] = sys->FeelDisk[k];
      st.planets.feelothers[k] = sys->FeelOthers[k];
      st.planets.binary[k] = sys->Binary[k];
    }
    prof.sigma_med = SigmaMed;
    prof.sigma_inf = SigmaInf;
    prof.energy_med = EnergyMed;
    prof.vtheta_med = VthetaMed;
    prof.vrad_med = VradMed;
    prof.global_soundspeed = GLOBAL_SoundSpeed;
    rc = fb_upload(g_ctx, &st, &prof);
    if (rc) dropin_fail("fb_upload", rc);
    if (MHDLSA && NBTURBMODES > 0) {
      /* the turbulent modes continue the drand48 stream where main.c left it */
      unsigned long long x = rand48_get();
      rc = fb_lsa_stream(g_ctx, &x, 1);
      if (rc) dropin_fail("fb_lsa_stream", rc);
    }
    if (NBPART != 0) {
      /* the particles as main.c left them, and the position of the drand48
         stream the turbulent kicks continue; the Gaussian generators have not
         been called before the first AlgoGas */
      dust_views(&dst, dsys);
      dst.rng_x = rand48_get();
      dst.kicks = 0;
      dst.particles_mass = Particles_Mass;
      rc = fb_dust_upload(g_ctx, &dst);
      if (rc) dropin_fail("fb_dust_upload", rc);
    }
  }
  rc = fb_algogas(g_ctx, &rep);
  if (rc && rc != FB_ERR_NEGATIVE) dropin_fail("fb_algogas", rc);  /* a crash is not fatal */
  g_substeps += rep.substeps;
  /* the scalars and the planets every DT; the fields only when a reference
     routine is about to read them (sync_host, called by the wrappers below) */
  rc = fb_download(g_ctx, &st, 0u);
  if (rc) dropin_fail("fb_download", rc);
  if (MHDLSA && NBTURBMODES > 0) {  /* the stream as the modes' draws left it */
    unsigned long long x = 0;
    rc = fb_lsa_stream(g_ctx, &x, 0);
    if (rc) dropin_fail("fb_lsa_stream", rc);
    rand48_set(x);
  }
  g_rho = Rho; g_vrad = Vrad; g_vtheta = Vtheta; g_energy = Energy; g_dsys = dsys;
  g_host_stale = 1;
  if (g_sync_always) sync_host();
  PhysicalTime = st.physical_time;
  OmegaFrame = st.omega_frame;  /* follows the planet in a corotating frame */
  LostMass = st.lost_mass;
  MINDT = st.mindt;
  MAXDT = st.maxdt;
  DiskOnPrimaryAcceleration.x = rep.disk_on_primary[0];
  DiskOnPrimaryAcceleration.y = rep.disk_on_primary[1];
  DiskOnPrimaryAcceleration_alt.x = rep.disk_on_primary_alt[0];
  DiskOnPrimaryAcceleration_alt.y = rep.disk_on_primary_alt[1];
  for (k = 0; k < 3; k++) {
    stardiscbarycenter_x[k] = st.stardiscbarycenter_x[k];
    stardiscbarycenter_y[k] = st.stardiscbarycenter_y[k];
  }
  for (k = 0; k < sys->nb; k++) {
    sys->mass[k] = st.planets.mass[k];
    sys->x[k] = st.planets.x[k];
    sys->y[k] = st.planets.y[k];
    sys->vx[k] = st.planets.vx[k];
    sys->vy[k] = st.planets.vy[k];
  }
  if (rep.crashes > 0 && g_crashes == 0) write_crash_dumps(Rho, Vrad, Vtheta, Energy);
  g_crashes = rep.crashes;
  /* one mark per substep as the reference prints them (SourceEuler.c:564-567):
     '.', or 'c' for a crashed substep */
  for (k = 0; k < rep.substeps - rep.crash_substeps; k++) masterprint(".");
  for (k = 0; k < rep.crash_substeps; k++) masterprint("c");
  masterprint("\n");
}

/* ---------------------------------------------------------------------------
 * The rest of the reference's time loop (main.c:302-397) reads the state
 * between AlgoGas calls only through the routines below.  Linked with
 * -Wl,--wrap=<name> for each of them (the drop-in build of oracle/Makefile
 * does so), the host fields are downloaded only when one of them is about to
 * read them (outputs, -a monitoring, Stockholm logs), and the two per-DT
 * planet logs are fed from the GPU instead:
 *   UpdateLog            the disc's force on each planet by fb_planet_force
 *                        (ComputeForce on the device density), written
 *                        exactly as src/Force.c:266-328 writes tqwk*.dat and
 *                        indtq*.dat;
 *   compute_selfgravity  the loop's logging call (DeltaT = 0, main.c:316,
 *                        which only computes the accelerations) on the GPU,
 *                        with the rings next to the planets brought back for
 *                        UpdateLogSG.
 * Before the first AlgoGas (no context yet) every wrapper calls the
 * reference's own routine.  FB_DROPIN_SYNC=1 in the environment downloads
 * every field after every DT instead. */
void __real_SendOutput();
void __real_UpdateLog();
void __real_UpdateLogStockholm();
void __real_compute_selfgravity();
void __real_CompareSGandSummationTorques();
void __real_WriteBarycentrePosition();
void __real_CheckMomentumConservation();
real __real_GasMomentum();
real __real_GasTotalMass();
real __real_GasTotalEnergy();
void __real_WriteDustSystemFile();
void __real_WriteJacobi();

void __wrap_SendOutput(int index, PolarGrid *dens, PolarGrid *gasvr, PolarGrid *gasvt, PolarGrid *gasenerg,
                       PolarGrid *label, PolarGrid *pcdens, PolarGrid *dustdens, PolarGrid *dustvr,
                       PolarGrid *dustvt, DustSystem *dsys)
{
  sync_host();
  __real_SendOutput(index, dens, gasvr, gasvt, gasenerg, label, pcdens, dustdens, dustvr, dustvt, dsys);
}

void __wrap_UpdateLog(Force *fc, PlanetarySystem *psys, PolarGrid *Rho, int outputnb, real time)
{
  int i, rc;
  real x, y, r, m, vx, vy, smoothing, f[8];
  FILE *out;
  char filename[MAX1D];
  if (!g_ctx || !g_host_stale) {
    __real_UpdateLog(fc, psys, Rho, outputnb, time);
    return;
  }
  for (i = 0; i < psys->nb; i++) {
    x = psys->x[i];
    y = psys->y[i];
    vx = psys->vx[i];
    vy = psys->vy[i];
    r = sqrt(x * x + y * y);
    m = psys->mass[i];
    if (RocheSmoothing)
      smoothing = r * pow(m / 3., 1. / 3.) * ROCHESMOOTHING;
    else
      smoothing = compute_smoothing(r);
    rc = fb_planet_force(g_ctx, x, y, smoothing, m, f);
    if (rc) dropin_fail("fb_planet_force", rc);
    fc->fx_inner = f[0]; fc->fx_ex_inner = f[1]; fc->fx_outer = f[2]; fc->fx_ex_outer = f[3];
    fc->fy_inner = f[4]; fc->fy_ex_inner = f[5]; fc->fy_outer = f[6]; fc->fy_ex_outer = f[7];
    sprintf(filename, "%stqwk%d.dat", OUTPUTDIR, i);
    out = fopen(filename, "a");
    if (out == NULL) {
      fprintf(stderr, "Can't open %s\n", filename);
      prs_exit(1);
    }
    fprintf(out, "%d\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\t%.18g\n", outputnb,
            x * fc->fy_inner - y * fc->fx_inner, x * fc->fy_outer - y * fc->fx_outer,
            x * fc->fy_ex_inner - y * fc->fx_ex_inner, x * fc->fy_ex_outer - y * fc->fx_ex_outer,
            vx * fc->fx_inner + vy * fc->fy_inner, vx * fc->fx_outer + vy * fc->fy_outer,
            vx * fc->fx_ex_inner + vy * fc->fy_ex_inner, vx * fc->fx_ex_outer + vy * fc->fy_ex_outer, time);
    fclose(out);
    sprintf(filename, "%sindtq%d.dat", OUTPUTDIR, i);
    out = fopen(filename, "a");
    if (out == NULL) {
      fprintf(stderr, "Can't open %s\n", filename);
      prs_exit(1);
    }
    fprintf(out, "%d\t%.18g\t%.18g\n", outputnb,
            -x * DiskOnPrimaryAcceleration.y + y * DiskOnPrimaryAcceleration.x, time);
    fclose(out);
  }
}

void __wrap_UpdateLogStockholm(PlanetarySystem *sys, PolarGrid *Rho, int outputnb, real time)
{
  sync_host();
  __real_UpdateLogStockholm(sys, Rho, outputnb, time);
}

void __wrap_compute_selfgravity(PolarGrid *Rho, PolarGrid *Vr, PolarGrid *Vt, PolarGrid *DVr, PolarGrid *DVt,
                                real DeltaT, boolean SGUpdate)
{
  int k, ip, lo, hi, rc;
  real rp;
  if (!g_ctx || DeltaT != 0.0 || SGZeroMode || !g_host_stale) {
    sync_host();
    __real_compute_selfgravity(Rho, Vr, Vt, DVr, DVt, DeltaT, SGUpdate);
    return;
  }
  /* the accelerations of the current density (compute_fftdensity and
     compute_sgacc, src/sgmain.c:23-28); the velocity update with DeltaT = 0
     changes nothing */
  rc = fb_stage(g_ctx, FB_STAGE_SELFGRAV, 0.0);
  if (rc) dropin_fail("fb_stage(SELFGRAV)", rc);
  if (CompareSGAndSummationTorques) {
    rc = fb_download_sgacc(g_ctx, 0, NRAD, gr->Field, gtheta->Field);
    if (rc) dropin_fail("fb_download_sgacc", rc);
  } else if (g_sys) {
    /* UpdateLogSG (src/Force.c:369-420) reads the rings ip-1 .. ip+1 around
       each planet inside the grid */
    for (k = 0; k < g_sys->nb; k++) {
      rp = sqrt(g_sys->x[k] * g_sys->x[k] + g_sys->y[k] * g_sys->y[k]);
      if (rp < Rinf[0] || rp >= Rsup[NRAD - 1]) continue;
      ip = 0;
      while (ip < NRAD && rp >= Rinf[ip]) ip++;
      ip--;
      lo = ip - 2 < 0 ? 0 : ip - 2;
      hi = ip + 2 > NRAD - 1 ? NRAD - 1 : ip + 2;
      rc = fb_download_sgacc(g_ctx, lo, hi - lo + 1, gr->Field, gtheta->Field);
      if (rc) dropin_fail("fb_download_sgacc", rc);
    }
  }
  SG_initcounter++;
}

void __wrap_CompareSGandSummationTorques(Force *force, PolarGrid *Rho, PlanetarySystem *sys)
{
  sync_host();
  __real_CompareSGandSummationTorques(force, Rho, sys);
}

void __wrap_WriteBarycentrePosition(PolarGrid *Rho)
{
  sync_host();
  __real_WriteBarycentrePosition(Rho);
}

void __wrap_CheckMomentumConservation(PolarGrid *Density, PolarGrid *Vtheta, PlanetarySystem *sys)
{
  sync_host();
  __real_CheckMomentumConservation(Density, Vtheta, sys);
}

real __wrap_GasMomentum(PolarGrid *Density, PolarGrid *Vtheta)
{
  sync_host();
  return __real_GasMomentum(Density, Vtheta);
}

real __wrap_GasTotalMass(PolarGrid *array)
{
  sync_host();
  return __real_GasTotalMass(array);
}

real __wrap_GasTotalEnergy(PolarGrid *Rho, PolarGrid *Vr, PolarGrid *Vt, PolarGrid *Energy)
{
  sync_host();
  return __real_GasTotalEnergy(Rho, Vr, Vt, Energy);
}

void __wrap_WriteDustSystemFile(DustSystem *dsys, int index)
{
  sync_host();
  __real_WriteDustSystemFile(dsys, index);
}

void __wrap_WriteJacobi(DustSystem *dsys, PlanetarySystem *sys, int k)
{
  sync_host();
  __real_WriteJacobi(dsys, sys, k);
}
