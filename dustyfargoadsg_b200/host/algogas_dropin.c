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

static fb_ctx *g_ctx = NULL;
static int g_crashes = 0;  /* AlreadyCrashed as last reported */

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
  if (OpenInner || NonReflecting || AccBoundary) p->unsupported |= FB_U_BOUNDARY;
  if (OuterSourceMass) p->unsupported |= FB_U_OUTERSOURCE;
  if (DampToViscous) p->unsupported |= FB_U_DAMPTOVISCOUS;
  if (AddMass) p->unsupported |= FB_U_ADDMASS;
  if (DiscEvaporation) p->unsupported |= FB_U_EVAPORATION;
  if (PhotoEvaporation) p->unsupported |= FB_U_PHOTOEVAP;
  if (SelfGravity && SGZeroMode) p->unsupported |= FB_U_SGZEROMODE;
  if (ZMPlus) p->unsupported |= FB_U_ZMPLUS;
  if (MHDLSA) p->unsupported |= FB_U_MHDLSA;
  if (EntropyDiffusion || RadiativeDiffusion) p->unsupported |= FB_U_THERMALDIFF;
  if (ThermalCooling) p->unsupported |= FB_U_THERMALCOOLING;
  if (TempPresc) p->unsupported |= FB_U_TEMPPRESC;
  if (Corotating) p->unsupported |= FB_U_COROTATING;
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
  if (!g_ctx) {
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
  rc = fb_download(g_ctx, &st, FB_F_ALL);
  if (rc) dropin_fail("fb_download", rc);
  if (EnergyEquation || Write_Temperature) fb_download_derived(g_ctx, 0, Temperature->Field);
  if (Write_Potential) fb_download_derived(g_ctx, 1, Potential->Field);
  PhysicalTime = st.physical_time;
  LostMass = st.lost_mass;
  MINDT = st.mindt;
  MAXDT = st.maxdt;
  for (k = 0; k < 3; k++) {
    stardiscbarycenter_x[k] = st.stardiscbarycenter_x[k];
    stardiscbarycenter_y[k] = st.stardiscbarycenter_y[k];
  }
  if (NBPART != 0) {
    dust_views(&dst, dsys);
    rc = fb_dust_download(g_ctx, &dst);
    if (rc) dropin_fail("fb_dust_download", rc);
    rand48_set(dst.rng_x);
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
