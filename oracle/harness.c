/* harness.c -- TEST INFRASTRUCTURE ONLY (the CPU oracle), never product code.
 *
 * Linked with the reference's own, unmodified objects (main.c included)
 * through `ld --wrap`, so that the reference's own main() (main.c:21-413)
 * drives the run.  The wrappers add, around reference functions that are
 * called across translation units:
 *
 *   InitGasDensity   (Pframeforce.c:297, called from main.c:164)
 *       after the reference fills Sigma(r), adds seeded white noise
 *       dens += A * SigmaMed[i] * (2u-1), u ~ drand48 seeded with ORACLE_SEED,
 *       in the reference's own loop order (Pframeforce.c:308-320), when
 *       ORACLE_NOISE=A is set.  The reference's AddNoise is fixed at 1e-3
 *       with a wall-clock seed (Pframeforce.c:317-320), which cannot express
 *       a seeded 1e-4 perturbation.
 *   AlgoGas          (SourceEuler.c:326, called from main.c:387)
 *       times each call (CLOCK_MONOTONIC), and writes a full-precision
 *       dump of the state after every ORACLE_DUMP_EVERY-th call into
 *       ORACLE_DUMP_DIR (plus the state before the first call).
 *       Built with -DFB_DROPIN the same wrapper instead calls the GPU
 *       drop-in (dustyfargoadsg_b200/host/algogas_dropin.c).
 *   Transport        (TransportEuler.c:65) counts substeps; with
 *       ORACLE_MAX_SUBSTEPS=K the run stops after K substeps (bounded CPU
 *       timing samples).  ORACLE_STAGE_DUMP=1 dumps the fields entering and
 *       leaving the first Transport, ComputeViscousTerms,
 *       UpdateVelocitiesWithViscosity, ApplyBoundaryCondition and
 *       EvanescentBoundary calls of the run.
 *       With ORACLE_NEGATE_ENERGY=l the energy of cell l changes sign
 *       before the first call (crash-report tests).
 *   DumpSources      (LowTasks.c:133) becomes a no-op (it shells out to cp).
 *
 * At exit it prints one line "ORACLE_TIMING {json}" on stderr with the
 * wall time spent inside AlgoGas, the substep count, cell-updates/s and the
 * wall time of the time loop from the first AlgoGas call to the end of the
 * last one (AlgoGas plus the loop's logs and outputs between the calls).
 *
 * Dump format ("FBD1"): one ASCII JSON header line, then raw little-endian
 * doubles.  The header lists {"name": [offset_in_doubles, count], ...} and
 * the grid size.
 */
#include "mp.h"
#include <sys/stat.h>

void __real_AlgoGas();
void __real_InitGasDensity();
void __real_Transport();
void __real_ComputeViscousTerms();
void __real_UpdateVelocitiesWithViscosity();
void __real_ApplyBoundaryCondition();
void __real_EvanescentBoundary();
#ifdef FB_DROPIN
long fb_dropin_substeps(void);
void fb_dropin_sync_host(void);
void fb_dropin_AlgoGas(Force *force, PolarGrid *Rho, PolarGrid *Vrad,
                       PolarGrid *Vtheta, PolarGrid *Energy, PolarGrid *Label,
                       PolarGrid *DRho, PolarGrid *dustpcdens,
                       PolarGrid *DVrad, PolarGrid *DVtheta,
                       PlanetarySystem *sys, DustSystem *dsys);
#endif

extern real LostMass;
extern boolean SelfGravity, SGZeroMode;

static double h_time_in_algogas = 0.0;
static double h_call_start = 0.0;
static double h_loop_start = -1.0, h_loop_end = 0.0;  /* first timed AlgoGas start, last AlgoGas end */
static long h_loop_calls0 = 0, h_loop_substeps0 = 0;
static long h_substeps = 0;
static long h_calls = 0;
static int h_atexit_set = 0;
static int h_stage_done = 0;
static int h_in_algogas = 0;

static double now_s(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void print_timing(void)
{
  double cells = (double)GLOBALNRAD * (double)NSEC;
  double rate = h_time_in_algogas > 0 ? (double)h_substeps * cells / h_time_in_algogas : 0.0;
  char line[512];
  FILE *f;
  const char *tf = getenv("ORACLE_TIMING_FILE");
  snprintf(line, sizeof line,
           "{\"wall_s\": %.9g, \"substeps\": %ld, \"algogas_calls\": %ld, "
           "\"nrad\": %d, \"nsec\": %d, \"cell_updates_per_s\": %.9g, \"loop_wall_s\": %.9g, "
           "\"loop_calls\": %ld, \"loop_substeps\": %ld}",
           h_time_in_algogas, h_substeps, h_calls, GLOBALNRAD, NSEC, rate,
           h_loop_start >= 0.0 ? h_loop_end - h_loop_start : 0.0, h_calls - h_loop_calls0,
           h_substeps - h_loop_substeps0);
  fprintf(stderr, "ORACLE_TIMING %s\n", line);
  if (tf && (f = fopen(tf, "w")) != NULL) {
    fprintf(f, "%s\n", line);
    fclose(f);
  }
}

static void ensure_atexit(void)
{
  if (!h_atexit_set) {
    atexit(print_timing);
    h_atexit_set = 1;
  }
}

/* ---------------------------------------------------------------- dumps */
#define MAXARR 48
typedef struct { const char *name; const real *p; long n; } darr;

static void write_dump(const char *path, darr *a, int na, double *sc, int nsc,
                       const char **scn)
{
  FILE *f = fopen(path, "wb");
  long off = 0;
  int k;
  if (!f) { fprintf(stderr, "harness: cannot write %s\n", path); exit(2); }
  fprintf(f, "{\"format\": \"FBD1\", \"nrad\": %d, \"nsec\": %d, \"arrays\": {",
          GLOBALNRAD, NSEC);
  for (k = 0; k < nsc; k++) {
    fprintf(f, "%s\"%s\": [%ld, 1]", (off ? ", " : ""), scn[k], off);
    off += 1;
  }
  for (k = 0; k < na; k++) {
    fprintf(f, "%s\"%s\": [%ld, %ld]", (off ? ", " : ""), a[k].name, off, a[k].n);
    off += a[k].n;
  }
  fprintf(f, "}}\n");
  fwrite(sc, sizeof(double), nsc, f);
  for (k = 0; k < na; k++) fwrite(a[k].p, sizeof(real), a[k].n, f);
  fclose(f);
}

/* Position of the libc drand48 stream (48-bit, exact in a double), read
   through seed48 and put back unchanged. */
static unsigned long long rand48_state(void)
{
  unsigned short probe[3] = {0, 0, 0}, keep[3];
  unsigned short *old = seed48(probe);
  keep[0] = old[0];
  keep[1] = old[1];
  keep[2] = old[2];
  seed48(keep);
  return (unsigned long long)keep[0] | ((unsigned long long)keep[1] << 16) | ((unsigned long long)keep[2] << 32);
}

static void dump_state(const char *tag, PolarGrid *Rho, PolarGrid *Vrad,
                       PolarGrid *Vtheta, PolarGrid *Energy,
                       PlanetarySystem *sys, DustSystem *dsys)
{
  const char *dir = getenv("ORACLE_DUMP_DIR");
  char path[1024];
  darr a[MAXARR];
  double sc[16];
  const char *scn[16];
  int na = 0, nsc = 0;
  long nf = (long)(NRAD + 1) * NSEC;
  if (!dir) return;
  mkdir(dir, 0755);
  snprintf(path, sizeof path, "%s/%s.fbd", dir, tag);
  scn[nsc] = "PhysicalTime"; sc[nsc++] = PhysicalTime;
  scn[nsc] = "OmegaFrame"; sc[nsc++] = OmegaFrame;
  scn[nsc] = "LostMass"; sc[nsc++] = LostMass;
  scn[nsc] = "MINDT"; sc[nsc++] = MINDT;
  scn[nsc] = "MAXDT"; sc[nsc++] = MAXDT;
  scn[nsc] = "substeps"; sc[nsc++] = (double)h_substeps;
  scn[nsc] = "nplanets"; sc[nsc++] = (double)(sys ? sys->nb : 0);
  scn[nsc] = "nbpart"; sc[nsc++] = (double)NBPART;
  scn[nsc] = "rng_state"; sc[nsc++] = (double)rand48_state();
  a[na].name = "dens"; a[na].p = Rho->Field; a[na++].n = nf;
  a[na].name = "vrad"; a[na].p = Vrad->Field; a[na++].n = nf;
  a[na].name = "vtheta"; a[na].p = Vtheta->Field; a[na++].n = nf;
  a[na].name = "energy"; a[na].p = Energy->Field; a[na++].n = nf;
  if (SoundSpeed) { a[na].name = "soundspeed"; a[na].p = SoundSpeed->Field; a[na++].n = nf; }
  if (Pressure) { a[na].name = "pressure"; a[na].p = Pressure->Field; a[na++].n = nf; }
  if (Potential) { a[na].name = "potential"; a[na].p = Potential->Field; a[na++].n = nf; }
  if (Temperature) { a[na].name = "temperature"; a[na].p = Temperature->Field; a[na++].n = nf; }
  if (DivergenceVelocity) { a[na].name = "divv"; a[na].p = DivergenceVelocity->Field; a[na++].n = nf; }
  if (ViscHeat) { a[na].name = "vischeat"; a[na].p = ViscHeat->Field; a[na++].n = nf; }
  a[na].name = "SigmaMed"; a[na].p = SigmaMed; a[na++].n = NRAD;
  a[na].name = "EnergyMed"; a[na].p = EnergyMed; a[na++].n = NRAD;
  a[na].name = "VthetaMed"; a[na].p = VthetaMed; a[na++].n = NRAD;
  a[na].name = "VradMed"; a[na].p = VradMed; a[na++].n = NRAD;
  a[na].name = "GLOBAL_SoundSpeed"; a[na].p = GLOBAL_SoundSpeed; a[na++].n = NRAD;
  a[na].name = "Radii"; a[na].p = Radii; a[na++].n = NRAD + 1;
  a[na].name = "Rmed"; a[na].p = Rmed; a[na++].n = NRAD;
  a[na].name = "Surf"; a[na].p = Surf; a[na++].n = NRAD;
  a[na].name = "stardiscbarycenter_x"; a[na].p = stardiscbarycenter_x; a[na++].n = 3;
  a[na].name = "stardiscbarycenter_y"; a[na].p = stardiscbarycenter_y; a[na++].n = 3;
  if (sys && sys->nb > 0) {
    a[na].name = "pl_mass"; a[na].p = sys->mass; a[na++].n = sys->nb;
    a[na].name = "pl_x"; a[na].p = sys->x; a[na++].n = sys->nb;
    a[na].name = "pl_y"; a[na].p = sys->y; a[na++].n = sys->nb;
    a[na].name = "pl_vx"; a[na].p = sys->vx; a[na++].n = sys->nb;
    a[na].name = "pl_vy"; a[na].p = sys->vy; a[na++].n = sys->nb;
  }
  if (SelfGravity && !SGZeroMode && gr && gtheta) {
    a[na].name = "sg_accr"; a[na].p = gr->Field; a[na++].n = nf;
    a[na].name = "sg_acct"; a[na].p = gtheta->Field; a[na++].n = nf;
  }
  if (dsys && NBPART > 0) {
    a[na].name = "pc_r"; a[na].p = dsys->r; a[na++].n = NBPART;
    a[na].name = "pc_th"; a[na].p = dsys->th; a[na++].n = NBPART;
    a[na].name = "pc_vr"; a[na].p = dsys->vr; a[na++].n = NBPART;
    a[na].name = "pc_vth"; a[na].p = dsys->vth; a[na++].n = NBPART;
    a[na].name = "pc_size"; a[na].p = dsys->dustsize; a[na++].n = NBPART;
    a[na].name = "pc_stokes"; a[na].p = dsys->stokesnb; a[na++].n = NBPART;
  }
  write_dump(path, a, na, sc, nsc, scn);
}

static void dump_fields(const char *tag, int n, const char **names, PolarGrid **g)
{
  const char *dir = getenv("ORACLE_DUMP_DIR");
  char path[1024];
  darr a[MAXARR];
  double sc[2];
  const char *scn[2] = {"PhysicalTime", "substeps"};
  long nf = (long)(NRAD + 1) * NSEC;
  int k;
  if (!dir) return;
  mkdir(dir, 0755);
  snprintf(path, sizeof path, "%s/%s.fbd", dir, tag);
  for (k = 0; k < n; k++) { a[k].name = names[k]; a[k].p = g[k]->Field; a[k].n = nf; }
  sc[0] = PhysicalTime;
  sc[1] = (double)h_substeps;
  write_dump(path, a, n, sc, 2, scn);
}

static int stage_dump_on(void)
{
  const char *s = getenv("ORACLE_STAGE_DUMP");
  return s && *s == '1' && h_stage_done == 0;
}

/* ------------------------------------------------------------ wrappers */
void __wrap_DumpSources(int argc, char *argv[], char *parfile, char *cfgfile)
{
  (void)argc; (void)argv; (void)parfile; (void)cfgfile;
}

void __wrap_InitGasDensity(PolarGrid *Rho)
{
  const char *amp_s = getenv("ORACLE_NOISE");
  const char *seed_s = getenv("ORACLE_SEED");
  __real_InitGasDensity(Rho);
  if (amp_s && atof(amp_s) != 0.0) {
    double amp = atof(amp_s);
    int i, j, nr = Rho->Nrad, ns = Rho->Nsec;
    real *dens = Rho->Field;
    oracle_libc_srand48(seed_s ? atol(seed_s) : 0L);
    for (i = 0; i < nr; i++)
      for (j = 0; j < ns; j++)
        dens[j + i * ns] += amp * SigmaMed[i] * (2.0 * drand48() - 1.0);
  }
}

void __wrap_Transport(PolarGrid *Rho, PolarGrid *Vrad, PolarGrid *Vtheta,
                      PolarGrid *Energy, PolarGrid *Label, real dt)
{
  const char *ms = getenv("ORACLE_MAX_SUBSTEPS");
  int stage = stage_dump_on();
  const char *nm[4] = {"dens", "vrad", "vtheta", "energy"};
  PolarGrid *g[4];
  g[0] = Rho; g[1] = Vrad; g[2] = Vtheta; g[3] = Energy;
  if (stage) dump_fields("stage_transport_in", 4, nm, g);
  __real_Transport(Rho, Vrad, Vtheta, Energy, Label, dt);
  if (stage) {
    dump_fields("stage_transport_out", 4, nm, g);
    {
      const char *dir = getenv("ORACLE_DUMP_DIR");
      char path[1024];
      FILE *f;
      if (dir) {
        snprintf(path, sizeof path, "%s/stage_transport_dt.txt", dir);
        if ((f = fopen(path, "w"))) { fprintf(f, "%.17g\n", dt); fclose(f); }
      }
    }
  }
  h_substeps++;
  if (ms && h_substeps >= atol(ms)) {
    h_time_in_algogas += now_s() - h_call_start;
    h_call_start = now_s();
    exit(0);
  }
}

void __wrap_ComputeViscousTerms(PolarGrid *Vr, PolarGrid *Vt, PolarGrid *Rho,
                                PolarGrid *DVr, PolarGrid *DVt, PolarGrid *DRho)
{
  int stage = stage_dump_on();
  const char *nm[3] = {"vrad", "vtheta", "dens"};
  PolarGrid *g[3];
  g[0] = Vr; g[1] = Vt; g[2] = Rho;
  if (stage && h_substeps == 0 && h_in_algogas) {
    static int once = 0;
    if (!once) { once = 1; dump_fields("stage_visc_in", 3, nm, g); }
  }
  __real_ComputeViscousTerms(Vr, Vt, Rho, DVr, DVt, DRho);
}

void __wrap_UpdateVelocitiesWithViscosity(PolarGrid *Vr, PolarGrid *Vt, PolarGrid *Rho,
                                          PolarGrid *DVr, PolarGrid *DVt, PolarGrid *DRho,
                                          real dt)
{
  int stage = stage_dump_on();
  const char *nm[3] = {"vrad", "vtheta", "dens"};
  PolarGrid *g[3];
  g[0] = Vr; g[1] = Vt; g[2] = Rho;
  __real_UpdateVelocitiesWithViscosity(Vr, Vt, Rho, DVr, DVt, DRho, dt);
  if (stage && h_substeps == 0 && h_in_algogas) {
    static int once = 0;
    if (!once) { once = 1; dump_fields("stage_visc_out", 3, nm, g); }
  }
}

void __wrap_ApplyBoundaryCondition(PolarGrid *Vrad, PolarGrid *Vtheta, PolarGrid *Rho,
                                   PolarGrid *Energy, PolarGrid *DVrad, PolarGrid *DVtheta,
                                   PolarGrid *DRho, real step, PlanetarySystem *sys)
{
  int stage = stage_dump_on();
  const char *nm[4] = {"dens", "vrad", "vtheta", "energy"};
  PolarGrid *g[4];
  g[0] = Rho; g[1] = Vrad; g[2] = Vtheta; g[3] = Energy;
  if (stage) dump_fields("stage_bc_in", 4, nm, g);
  __real_ApplyBoundaryCondition(Vrad, Vtheta, Rho, Energy, DVrad, DVtheta, DRho, step, sys);
  if (stage) dump_fields("stage_bc_out", 4, nm, g);
}

void __wrap_EvanescentBoundary(PolarGrid *Vrad, PolarGrid *Vtheta, PolarGrid *Rho,
                               PolarGrid *Energy, PolarGrid *DVrad, PolarGrid *DVtheta,
                               PolarGrid *DRho, real step)
{
  int stage = stage_dump_on();
  const char *nm[4] = {"dens", "vrad", "vtheta", "energy"};
  PolarGrid *g[4];
  g[0] = Rho; g[1] = Vrad; g[2] = Vtheta; g[3] = Energy;
  __real_EvanescentBoundary(Vrad, Vtheta, Rho, Energy, DVrad, DVtheta, DRho, step);
  if (stage) {
    dump_fields("stage_damp_out", 4, nm, g);
    h_stage_done = 1;
  }
}

void __wrap_AlgoGas(Force *force, PolarGrid *Rho, PolarGrid *Vrad,
                    PolarGrid *Vtheta, PolarGrid *Energy, PolarGrid *Label,
                    PolarGrid *DRho, PolarGrid *dustpcdens, PolarGrid *DVrad,
                    PolarGrid *DVtheta, PlanetarySystem *sys, DustSystem *dsys)
{
  const char *ev = getenv("ORACLE_DUMP_EVERY");
  long every = ev ? atol(ev) : 1;
  char tag[64];
  ensure_atexit();
  if (h_calls == 0) {
    /* ORACLE_NEGATE_ENERGY=l flips the sign of the energy of cell l before
       the first DT: the input of the crash-report tests (DetectCrash,
       SourceEuler.c:545-566) */
    const char *neg = getenv("ORACLE_NEGATE_ENERGY");
    if (neg) Energy->Field[atol(neg)] = -Energy->Field[atol(neg)];
    dump_state("state_init", Rho, Vrad, Vtheta, Energy, sys, dsys);
  }
  h_call_start = now_s();
  {
    /* ORACLE_TIMING_SKIP=W starts the loop clock at call W (warm-up calls) */
    const char *sk = getenv("ORACLE_TIMING_SKIP");
    if (h_loop_start < 0.0 && h_calls >= (sk ? atol(sk) : 0L)) {
      h_loop_start = h_call_start;
      h_loop_calls0 = h_calls;
      h_loop_substeps0 = h_substeps;
    }
  }
  h_in_algogas = 1;
#ifdef FB_DROPIN
  fb_dropin_AlgoGas(force, Rho, Vrad, Vtheta, Energy, Label, DRho, dustpcdens,
                    DVrad, DVtheta, sys, dsys);
#else
  __real_AlgoGas(force, Rho, Vrad, Vtheta, Energy, Label, DRho, dustpcdens,
                 DVrad, DVtheta, sys, dsys);
#endif
  h_loop_end = now_s();
  h_time_in_algogas += h_loop_end - h_call_start;
  h_in_algogas = 0;
  h_calls++;
#ifdef FB_DROPIN
  h_substeps = fb_dropin_substeps();  /* the drop-in's count: Transport is not called */
#endif
  if (every > 0 && (h_calls % every) == 0) {
    snprintf(tag, sizeof tag, "state_%05ld", h_calls);
#ifdef FB_DROPIN
    fb_dropin_sync_host();  /* the drop-in brings fields back only on demand */
#endif
    dump_state(tag, Rho, Vrad, Vtheta, Energy, sys, dsys);
  }
}
