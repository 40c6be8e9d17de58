/* fb_host.c -- host side of libfargo_b200.so: .par parameters, planet
 * configuration, 1-D geometry and initial conditions.
 *
 * This is the part of the reference's driver that the GPU step depends on,
 * restated in C with the reference's own expressions and evaluation order so
 * that the initial state is bit-identical to the reference's sequential
 * build (glibc libm supplies exp/log/pow/sqrt/sin/cos on both sides).
 */
#define _GNU_SOURCE
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fb_internal.h"

/* ------------------------------------------------------------------ rand48 */
/* POSIX drand48: 48-bit LCG X <- (a X + c) mod 2^48 with a = 0x5DEECE66D,
 * c = 0xB; srand48(s) sets X = (s mod 2^32) << 16 | 0x330E; drand48 returns
 * X * 2^-48.  Used for the seeded initial noise. */
void fb_srand48(fb_rand48 *s, long seed)
{
  s->x = (((unsigned long long)(unsigned int)seed) << 16) | 0x330Eull;
}

double fb_drand48(fb_rand48 *s)
{
  s->x = (0x5DEECE66Dull * s->x + 0xBull) & 0xFFFFFFFFFFFFull;
  return ldexp((double)s->x, -48);
}

unsigned long long fb_rand48_state(long seed, long long draws)
{
  fb_rand48 r;
  fb_srand48(&r, seed);
  for (long long n = 0; n < draws; n++) r.x = (0x5DEECE66Dull * r.x + 0xBull) & 0xFFFFFFFFFFFFull;
  return r.x;
}

/* ---------------------------------------------------------------- defaults */
int fb_params_default(fb_params *p)
{
  if (!p) return FB_ERR_INVALID;
  memset(p, 0, sizeof *p);
  /* src/var.c:13-202 defaults */
  p->dt = 1.0;
  p->sigma0 = 173.0;
  p->ninterm = 10;
  p->ntot = 1501;
  p->nrad = 64;
  p->nsec = 64;
  p->rmin = 1.0;
  p->rmax = 1.0;
  p->log_grid = 0;                 /* RADIALSPACING "ARITHMETIC" */
  p->pmin = 0.0;
  p->pmax = 6.2831853071795864;
  p->thicknesssmoothing = 0.3;
  p->sgthicknesssmoothing = 0.3;
  p->rochesmoothing = 0.0;
  p->indirecttermsmoothing = 0.0;
  p->aspectratio = 0.05;
  p->viscosity = 0.0;
  p->alphaviscosity = 0.0;
  p->sigmaslope = 0.0;
  p->omegaframe = 0.0;
  p->masstaper = 0.0000001;
  p->flaringindex = 0.0;
  p->eccentricity = 0.0;
  p->excludehillfactor = 1.0;
  p->imposeddiskdrift = 0.0;
  p->adiabaticindex = 1.4;
  p->betacoolingtime = 10.0;
  p->betacoolingslope = 0.0;
  p->thermal_cooling = 0;          /* THERMALCOOLING NO, SETCONSTANTOPACITY NO */
  p->constant_opacity = 0;
  p->imposedconstantopacity = 0.1; /* src/var.c:193-195 */
  p->factoropacities = 1.0;
  p->stellar_irradiation = 0;          /* src/var.c:88-91 */
  p->backgroundtemperature = 50.0;
  p->slopebackgroundtemperature = -0.5;
  p->stellarluminosity = 1.0;
  p->dampingtodynamicaltimeratio = 0.3;
  p->wkzrmin = 0.0;
  p->wkzrmax = 0.0;
  p->densityfloor = 1e-9;
  p->mindt = 100.0;
  p->maxdt = 0.00001;
  p->releasedate = 0.0;
  p->releaseradius = 0.0;
  p->factorunitmass = 1.0;
  p->factorunitlength = 1.0;
  p->factormmw = 1.0;
  p->sizeminpart = 0.001;
  p->sizemaxpart = 0.001;
  p->sizepartslope = 3.0;
  p->rhopart = 1.0;
  p->nbpart = 0;
  p->dustslope = 0.5;
  p->rmindust = 0.0;
  p->rmaxdust = 0.0;
  /* src/Interpret.c:23-50 boolean defaults */
  p->fast_transport = 1;
  p->indirect_term = 1;
  p->discard_gas_indirect_term = 0;
  p->alternative_gas_indirect_term = 0;
  p->wall_boundary = 1;            /* INNERBOUNDARY "WALL" */
  p->evanescent = 0;
  p->energy_equation = 0;
  p->viscous_heating = 1;
  p->beta_cooling = 0;
  p->self_gravity = 0;
  p->forced_circular = 0;
  p->exclude_hill = 0;
  p->damp_to_axi = 1;
  p->damp_to_ini = 0;
  p->add_floors = 1;
  p->zero_vrad_bc = 0;
  p->open_inner = 0;
  p->kn_open = 0;
  p->non_reflecting = 0;
  p->dust_feel_disk = 1;
  p->dust_feel_planets = 1;
  p->dust_feel_turb = 0;
  p->dust_feedback = 0;
  p->dust_feel_sg = 1;
  p->sfta = 1;
  p->write_dust_density = 0;
  p->interpolation = 2;
  strcpy(p->planetconfig, "Systems/SolarSystem.cfg");
  strcpy(p->outputdir, "~masset");
  /* turbulent potential (src/var.c:70-72, 99-102, 133-134) */
  p->mhd_lsa = 0;
  p->nbturbmodes = 50;
  p->high_m_cutoff = 0;
  p->gammaturb = 0.00001;
  p->lsamodespeedup = 0.1;
  p->turbrmin = 0.0;
  p->turbrmax = 0.0;
  p->cavityradius = 0.0;
  p->cavityratio = 1.0;
  p->cavitywidth = 1.0;
  /* thermal diffusion (src/var.c:85-86, 93) */
  p->entropy_diffusion = 0;
  p->radiative_diffusion = 0;
  p->diffusivity = 0.000001;
  p->corotating = 0;
  p->add_noise = 0;
  p->temppresc = 0;
  p->presctime0 = 6.28;  /* src/var.c:95 */
  return FB_OK;
}

/* ------------------------------------------------------------- .par reader */
typedef struct {
  char key[80];
  double num;
  char str[290];
} kv_t;

typedef struct {
  kv_t *v;
  int n, cap;
} kvset_t;

static kv_t *kv_find(kvset_t *s, const char *key)
{
  int i;
  for (i = 0; i < s->n; i++)
    if (strcmp(s->v[i].key, key) == 0) return &s->v[i];
  return NULL;
}

static double kv_num(kvset_t *s, const char *key, double dflt)
{
  kv_t *k = kv_find(s, key);
  return k ? k->num : dflt;
}

static int kv_int(kvset_t *s, const char *key, int dflt)
{
  kv_t *k = kv_find(s, key);
  return k ? (int)k->num : dflt;
}

/* first character of a string switch, or the default's first character */
static char kv_c(kvset_t *s, const char *key, char dflt)
{
  kv_t *k = kv_find(s, key);
  return k ? k->str[0] : dflt;
}

static int is_c(char c, char up) { return c == up || c == (char)tolower((unsigned char)up); }

int fb_params_read_par(fb_params *p, const char *path)
{
  static const char *necessary[] = {"DT", "SIGMA0", "NINTERM", "NTOT", "OUTPUTDIR",
                                    "NRAD", "NSEC", "RMIN", "RMAX", "ASPECTRATIO",
                                    "SIGMASLOPE", "ADIABATICINDEX", NULL};
  FILE *f;
  char s[350], nm[300], stringval[290];
  double temp = 0.0;
  kvset_t set = {NULL, 0, 0};
  int i, ok = FB_OK;
  char c;
  if (!p || !path) return FB_ERR_INVALID;
  fb_params_default(p);
  f = fopen(path, "r");
  if (!f) return FB_ERR_IO;
  /* line rules of ReadVariables (src/Interpret.c:101-135) */
  while (fgets(s, 349, f) != NULL) {
    char *s1;
    kv_t *k;
    int success = sscanf(s, "%299s ", nm);
    if (success != 1 || nm[0] == '#') continue;
    s1 = s + strlen(nm);
    stringval[0] = 0;
    sscanf(s1 + strspn(s1, "\t :=>_"), "%lf", &temp);
    sscanf(s1 + strspn(s1, "\t :=>_"), "%289s ", stringval);
    for (i = 0; nm[i]; i++) nm[i] = (char)toupper((unsigned char)nm[i]);
    k = kv_find(&set, nm);
    if (!k) {
      if (set.n == set.cap) {
        set.cap = set.cap ? 2 * set.cap : 64;
        set.v = (kv_t *)realloc(set.v, sizeof(kv_t) * set.cap);
        if (!set.v) { fclose(f); return FB_ERR_NOMEM; }
      }
      k = &set.v[set.n++];
      snprintf(k->key, sizeof k->key, "%s", nm);
    }
    k->num = temp;
    snprintf(k->str, sizeof k->str, "%s", stringval);
  }
  fclose(f);
  for (i = 0; necessary[i]; i++)
    if (!kv_find(&set, necessary[i])) ok = FB_ERR_INVALID;

  p->dt = kv_num(&set, "DT", p->dt);
  p->sigma0 = kv_num(&set, "SIGMA0", p->sigma0);
  p->ninterm = kv_int(&set, "NINTERM", p->ninterm);
  p->ntot = kv_int(&set, "NTOT", p->ntot);
  p->nrad = kv_int(&set, "NRAD", p->nrad);
  p->nsec = kv_int(&set, "NSEC", p->nsec);
  p->rmin = kv_num(&set, "RMIN", p->rmin);
  p->rmax = kv_num(&set, "RMAX", p->rmax);
  p->pmin = kv_num(&set, "PMIN", p->pmin);
  p->pmax = kv_num(&set, "PMAX", p->pmax);
  p->thicknesssmoothing = kv_num(&set, "THICKNESSSMOOTHING", p->thicknesssmoothing);
  p->sgthicknesssmoothing = kv_num(&set, "SGTHICKNESSSMOOTHING", p->sgthicknesssmoothing);
  p->rochesmoothing = kv_num(&set, "ROCHESMOOTHING", p->rochesmoothing);
  p->indirecttermsmoothing = kv_num(&set, "INDIRECTTERMSMOOTHING", p->indirecttermsmoothing);
  p->aspectratio = kv_num(&set, "ASPECTRATIO", p->aspectratio);
  p->viscosity = kv_num(&set, "VISCOSITY", p->viscosity);
  p->alphaviscosity = kv_num(&set, "ALPHAVISCOSITY", p->alphaviscosity);
  p->sigmaslope = kv_num(&set, "SIGMASLOPE", p->sigmaslope);
  p->omegaframe = kv_num(&set, "OMEGAFRAME", p->omegaframe);
  p->masstaper = kv_num(&set, "MASSTAPER", p->masstaper);
  p->flaringindex = kv_num(&set, "FLARINGINDEX", p->flaringindex);
  p->eccentricity = kv_num(&set, "ECCENTRICITY", p->eccentricity);
  p->excludehillfactor = kv_num(&set, "EXCLUDEHILLFACTOR", p->excludehillfactor);
  p->imposeddiskdrift = kv_num(&set, "IMPOSEDDISKDRIFT", p->imposeddiskdrift);
  p->adiabaticindex = kv_num(&set, "ADIABATICINDEX", p->adiabaticindex);
  p->betacoolingtime = kv_num(&set, "BETACOOLINGTIME", p->betacoolingtime);
  p->betacoolingslope = kv_num(&set, "BETACOOLINGSLOPE", p->betacoolingslope);
  p->imposedconstantopacity = kv_num(&set, "IMPOSEDCONSTANTOPACITY", p->imposedconstantopacity);
  p->factoropacities = kv_num(&set, "FACTOROPACITIES", p->factoropacities);
  p->backgroundtemperature = kv_num(&set, "BACKGROUNDTEMPERATURE", p->backgroundtemperature);
  p->slopebackgroundtemperature = kv_num(&set, "SLOPEBACKGROUNDTEMPERATURE", p->slopebackgroundtemperature);
  p->stellarluminosity = kv_num(&set, "STELLARLUMINOSITY", p->stellarluminosity);
  p->dampingtodynamicaltimeratio = kv_num(&set, "DAMPINGTODYNAMICALTIMERATIO", p->dampingtodynamicaltimeratio);
  p->wkzrmin = kv_num(&set, "WKZRMIN", p->wkzrmin);
  p->wkzrmax = kv_num(&set, "WKZRMAX", p->wkzrmax);
  p->densityfloor = kv_num(&set, "DENSITYFLOOR", p->densityfloor);
  p->mindt = kv_num(&set, "MINDT", p->mindt);
  p->maxdt = kv_num(&set, "MAXDT", p->maxdt);
  p->releasedate = kv_num(&set, "RELEASEDATE", p->releasedate);
  p->releaseradius = kv_num(&set, "RELEASERADIUS", p->releaseradius);
  p->factorunitmass = kv_num(&set, "FACTORUNITMASS", p->factorunitmass);
  p->factorunitlength = kv_num(&set, "FACTORUNITLENGTH", p->factorunitlength);
  p->factormmw = kv_num(&set, "FACTORMMW", p->factormmw);
  p->sizeminpart = kv_num(&set, "SIZEMINPART", p->sizeminpart);
  p->sizemaxpart = kv_num(&set, "SIZEMAXPART", p->sizemaxpart);
  p->sizepartslope = kv_num(&set, "SIZEPARTSLOPE", p->sizepartslope);
  p->rhopart = kv_num(&set, "RHOPART", p->rhopart);
  p->nbpart = kv_int(&set, "NBPART", p->nbpart);
  p->dustslope = kv_num(&set, "DUSTSLOPE", p->dustslope);
  p->rmindust = kv_num(&set, "RMINDUST", p->rmindust);
  p->rmaxdust = kv_num(&set, "RMAXDUST", p->rmaxdust);
  {
    kv_t *k = kv_find(&set, "PLANETCONFIG");
    if (k) snprintf(p->planetconfig, sizeof p->planetconfig, "%s", k->str);
    k = kv_find(&set, "OUTPUTDIR");
    if (k) snprintf(p->outputdir, sizeof p->outputdir, "%s", k->str);
  }

  /* String switches, decoded by first letter (src/Interpret.c:165-479). */
  c = kv_c(&set, "RADIALSPACING", 'A');
  p->log_grid = is_c(c, 'L');
  c = kv_c(&set, "TRANSPORT", 'F');
  if (is_c(c, 'S')) p->fast_transport = 0;
  c = kv_c(&set, "INNERBOUNDARY", 'W');
  p->wall_boundary = is_c(c, 'W');
  p->open_inner = is_c(c, 'O') || is_c(c, 'K');
  p->kn_open = is_c(c, 'K');
  p->non_reflecting = is_c(c, 'N');
  if (is_c(c, 'A')) p->unsupported |= FB_U_BOUNDARY;  /* the accreting boundary is not built */
  c = kv_c(&set, "WAVEKILLINGZONES", 'N');
  p->evanescent = is_c(c, 'Y');
  if (is_c(kv_c(&set, "DAMPTOINI", 'N'), 'Y')) { p->damp_to_ini = 1; p->damp_to_axi = 0; }
  if (is_c(kv_c(&set, "DAMPTOAXI", 'Y'), 'N')) { p->damp_to_axi = 0; p->damp_to_ini = 1; }
  if (is_c(kv_c(&set, "DAMPTOVISCOUS", 'N'), 'Y')) p->unsupported |= FB_U_DAMPTOVISCOUS;
  if (is_c(kv_c(&set, "ADDFLOORS", 'Y'), 'N')) p->add_floors = 0;
  if (is_c(kv_c(&set, "ZEROVRADBC", 'N'), 'Y')) p->zero_vrad_bc = 1;
  if (is_c(kv_c(&set, "INDIRECTTERM", 'Y'), 'N')) p->indirect_term = 0;
  if (is_c(kv_c(&set, "DISCARDGASINDIRECTTERM", 'N'), 'Y')) p->discard_gas_indirect_term = 1;
  if (is_c(kv_c(&set, "ALTERNATIVEGASINDIRECTTERM", 'N'), 'Y')) p->alternative_gas_indirect_term = 1;
  c = kv_c(&set, "SELFGRAVITY", 'N');
  if (is_c(c, 'Y')) p->self_gravity = 1;
  if (is_c(c, 'Z')) { p->self_gravity = 1; p->unsupported |= FB_U_SGZEROMODE; }
  if (is_c(kv_c(&set, "ZMPLUS", 'N'), 'Y') && is_c(c, 'Z')) p->unsupported |= FB_U_ZMPLUS;
  if (is_c(kv_c(&set, "ENERGYEQUATION", 'N'), 'Y')) p->energy_equation = 1;
  if (p->energy_equation && p->adiabaticindex == 1) p->energy_equation = 0; /* Interpret.c:426-429 */
  if (is_c(kv_c(&set, "VISCOUSHEATING", 'Y'), 'N')) p->viscous_heating = 0;
  if (is_c(kv_c(&set, "BETACOOLING", 'N'), 'Y')) p->beta_cooling = 1;
  /* thermal diffusion (src/Interpret.c:381-388); the implicit solver's
     red-black sweep equals the reference's sequential one only when the
     two cells either side of the azimuthal wrap have different colours */
  if (is_c(kv_c(&set, "ENTROPYDIFFUSION", 'N'), 'Y')) p->entropy_diffusion = 1;
  c = kv_c(&set, "RADIATIVEDIFFUSION", 'N');
  if (is_c(c, 'E')) p->radiative_diffusion = 1;
  if (is_c(c, 'I')) p->radiative_diffusion = 2;
  p->diffusivity = kv_num(&set, "DIFFUSIVITY", p->diffusivity);
  if (p->radiative_diffusion == 2 && (p->nsec % 2) != 0) p->unsupported |= FB_U_THERMALDIFF;
  if (is_c(kv_c(&set, "THERMALCOOLING", 'N'), 'Y')) p->thermal_cooling = 1;
  if (is_c(kv_c(&set, "SETCONSTANTOPACITY", 'N'), 'Y')) p->constant_opacity = 1;
  c = kv_c(&set, "STELLARIRRADIATION", 'N');
  if (is_c(c, 'Y')) p->stellar_irradiation = 1;
  if (is_c(c, 'L')) p->stellar_irradiation = 2;
  if (is_c(kv_c(&set, "TEMPPRESC", 'N'), 'Y')) p->temppresc = 1;  /* Interpret.c:397 */
  p->presctime0 = kv_num(&set, "PRESCTIME0", p->presctime0);
  if (is_c(kv_c(&set, "FORCEDCIRCULAR", 'N'), 'Y')) p->forced_circular = 1;
  if (is_c(kv_c(&set, "FORCEDINNERCIRCULAR", 'N'), 'Y')) p->unsupported |= FB_U_FORCEDINNER;
  if (is_c(kv_c(&set, "EXCLUDEHILL", 'N'), 'Y')) p->exclude_hill = 1;
  c = kv_c(&set, "FRAME", 'F');
  if (is_c(c, 'C')) p->corotating = 1;  /* Interpret.c:225-232 */
  if (is_c(c, 'G') || is_c(c, 'B')) p->unsupported |= FB_U_COROTATING;
  if (p->corotating && is_c(kv_c(&set, "COROTATEWITHOUTERPLANET", 'N'), 'Y')) p->unsupported |= FB_U_COROTATING;
  if (is_c(kv_c(&set, "CICPLANET", 'N'), 'Y')) p->unsupported |= FB_U_CICPLANET;
  if (is_c(kv_c(&set, "BM08TRICK", 'N'), 'Y')) p->unsupported |= FB_U_BM08;
  if (is_c(kv_c(&set, "COMPUTECPDMASS", 'N'), 'Y')) p->unsupported |= FB_U_CPDMASS;
  if (is_c(kv_c(&set, "LABELADVECTION", 'N'), 'Y')) p->unsupported |= FB_U_LABEL;
  if (is_c(kv_c(&set, "IMPOSEDDENSITY", 'N'), 'Y')) p->unsupported |= FB_U_IMPOSEDDENSITY;
  c = kv_c(&set, "ADDM1", 'N');
  if (is_c(c, 'Y') || is_c(c, 'B')) p->unsupported |= FB_U_ADDM;
  if (is_c(kv_c(&set, "ADDM2", 'N'), 'Y')) p->unsupported |= FB_U_ADDM;
  if (is_c(kv_c(&set, "ADDM1TOM10", 'N'), 'Y')) p->unsupported |= FB_U_ADDM;
  if (is_c(kv_c(&set, "ADDNOISE", 'N'), 'Y')) p->add_noise = 1;  /* Interpret.c:373-376 */
  c = kv_c(&set, "TAILOFF", 'N');
  if (is_c(c, 'G') || is_c(c, 'H') || is_c(c, 'E') || is_c(c, 'A') || is_c(c, 'B') ||
      is_c(c, 'S') || is_c(c, 'I'))
    p->unsupported |= FB_U_TAILOFF;
  if (is_c(kv_c(&set, "CAVITYTORQUE", 'N'), 'Y')) p->unsupported |= FB_U_CENTRIFUGAL;
  if (is_c(kv_c(&set, "DUSTFLUID", 'N'), 'Y')) p->unsupported |= FB_U_DUSTFLUID;
  if (is_c(kv_c(&set, "OUTERSOURCEMASS", 'N'), 'Y')) p->unsupported |= FB_U_OUTERSOURCE;
  if (is_c(kv_c(&set, "ADDMASS", 'N'), 'Y')) p->unsupported |= FB_U_ADDMASS;
  if (is_c(kv_c(&set, "DISCEVAPORATION", 'N'), 'Y')) p->unsupported |= FB_U_EVAPORATION;
  if (is_c(kv_c(&set, "PHOTOEVAPORATION", 'N'), 'Y')) p->unsupported |= FB_U_PHOTOEVAP;
  /* MHD L: the turbulent potential (src/Interpret.c:404-410); it draws from
     the drand48 stream the particles' kicks and initial draws share, so the
     two together are refused */
  p->nbturbmodes = kv_int(&set, "NBTURBMODES", p->nbturbmodes);
  p->gammaturb = kv_num(&set, "GAMMATURB", p->gammaturb);
  p->lsamodespeedup = kv_num(&set, "LSAMODESPEEDUP", p->lsamodespeedup);
  p->turbrmin = kv_num(&set, "TURBRMIN", p->turbrmin);
  p->turbrmax = kv_num(&set, "TURBRMAX", p->turbrmax);
  p->cavityradius = kv_num(&set, "CAVITYRADIUS", p->cavityradius);
  p->cavityratio = kv_num(&set, "CAVITYRATIO", p->cavityratio);
  p->cavitywidth = kv_num(&set, "CAVITYWIDTH", p->cavitywidth);
  if (is_c(kv_c(&set, "HIGHMCUTOFF", 'N'), 'Y')) p->high_m_cutoff = 1;
  if (is_c(kv_c(&set, "MHD", 'N'), 'L')) {
    p->mhd_lsa = 1;
    if (p->nbturbmodes < 0 || p->nbturbmodes > FB_LSA_MAX_MODES || p->nbpart > 0) p->unsupported |= FB_U_MHDLSA;
  }
  if (kv_num(&set, "CAVITYRADIUS", 0.0) != 0.0 || kv_num(&set, "CAVITYRATIO", 1.0) != 1.0)
    p->unsupported |= FB_U_CAVITY;
  if (kv_num(&set, "TRANSITIONRADIUS", 0.0) != 0.0 || kv_num(&set, "TRANSITIONRATIO", 1.0) != 1.0)
    p->unsupported |= FB_U_TRANSITION;
  if (kv_num(&set, "LAMBDADOUBLING", 0.0) != 0.0) p->unsupported |= FB_U_LAMBDADOUBLING;
  if (p->releasedate != 0.0) p->unsupported |= FB_U_RELEASE;
  if (kv_num(&set, "RELEASEDATEVISCOSITY", 0.0) > 1e-3) p->unsupported |= FB_U_VISCRELEASE;
  /* dust particles */
  if (is_c(kv_c(&set, "DUSTFEELDISK", 'Y'), 'N')) p->dust_feel_disk = 0;
  if (is_c(kv_c(&set, "DUSTFEELPLANETS", 'Y'), 'N')) p->dust_feel_planets = 0;
  c = kv_c(&set, "DUSTFEELTURB", 'N');
  if (is_c(c, 'Y') || is_c(c, 'C')) p->dust_feel_turb = 1;
  if (is_c(kv_c(&set, "DUSTFEEDBACK", 'N'), 'Y')) p->dust_feedback = 1;
  if (is_c(kv_c(&set, "SFTAPPROX", 'Y'), 'N')) p->sfta = 0;
  c = kv_c(&set, "INTERPOLATION", 'T');
  if (is_c(c, 'N')) p->interpolation = 0;
  if (is_c(c, 'C')) p->interpolation = 1;
  if (is_c(c, 'T')) p->interpolation = 2;
  if (p->nbpart != 0 && is_c(kv_c(&set, "NODTCONSTRAINTBYPCS", 'Y'), 'N'))
    p->unsupported |= FB_U_DUSTTIMESTEP;
  if (p->nbpart != 0) {
    /* particle options outside this build */
    if (is_c(kv_c(&set, "ZZINTEGRATOR", 'N'), 'Y')) p->unsupported |= FB_U_ZZINTEGRATOR;
    if (is_c(kv_c(&set, "DUSTGROWTH", 'N'), 'Y')) p->unsupported |= FB_U_DUSTGROWTH;
    if (is_c(kv_c(&set, "REMOVEDUSTFROMPLANETSHILLRADIUS", 'N'), 'Y')) p->unsupported |= FB_U_HILLREMOVAL;
    if (p->interpolation != 2) p->unsupported |= FB_U_INTERPOLATION;
    if (is_c(kv_c(&set, "DUSTFEELSG", 'Y'), 'Z')) p->unsupported |= FB_U_DUSTSGZERO;
    if (p->omegaframe != 0.0 || p->corotating) p->unsupported |= FB_U_COROTATING;
  }
  if (is_c(kv_c(&set, "DUSTFEELSG", 'Y'), 'N')) p->dust_feel_sg = 0;
  if (!is_c(kv_c(&set, "WRITEDUSTDENSITY", 'N'), 'N')) p->write_dust_density = 1;  /* Interpret.c:255-258 */
  if (p->nbpart != 0 && p->self_gravity && is_c(kv_c(&set, "SOFTWRITING", 'N'), 'Y'))
    p->unsupported |= FB_U_SOFTWRITING;
  if (p->alphaviscosity != 0.0 && p->viscosity != 0.0) ok = FB_ERR_INVALID; /* Interpret.c:453-459 */
  if (p->self_gravity && p->sgthicknesssmoothing == 0.0) ok = FB_ERR_INVALID;
  if (p->evanescent && (p->wkzrmin == 0.0 || p->wkzrmax == 0.0)) ok = FB_ERR_INVALID;
  if (p->excludehillfactor < 0.0 || p->excludehillfactor > 1.0) ok = FB_ERR_INVALID;
  if (p->nrad < 4 || p->nsec < 2) ok = FB_ERR_INVALID;
  free(set.v);
  return ok;
}

const char *fb_unsupported_name(const fb_params *p)
{
  static const struct { unsigned long long bit; const char *name; } names[] = {
    {FB_U_CENTRIFUGAL, "CentrifugalBalance/CavityTorque"}, {FB_U_TAILOFF, "TailOff"},
    {FB_U_DUSTFLUID, "DustFluid"}, {FB_U_BOUNDARY, "InnerBoundary Accreting"},
    {FB_U_OUTERSOURCE, "OuterSourceMass"}, {FB_U_DAMPTOVISCOUS, "DampToViscous"},
    {FB_U_ADDMASS, "AddMass"}, {FB_U_EVAPORATION, "DiscEvaporation"},
    {FB_U_PHOTOEVAP, "PhotoEvaporation"}, {FB_U_SGZEROMODE, "SelfGravity Z (zero mode)"},
    {FB_U_ZMPLUS, "ZMPlus"}, {FB_U_MHDLSA, "MHD LSA turbulence"},
    {FB_U_THERMALDIFF, "Entropy/radiative diffusion"}, {FB_U_THERMALCOOLING, "ThermalCooling"}, {FB_U_IRRADIATION, "StellarIrradiation"},
    {FB_U_TEMPPRESC, "TempPresc"}, {FB_U_COROTATING, "Corotating frame"},
    {FB_U_CICPLANET, "CICPlanet"}, {FB_U_BM08, "BM08Trick"}, {FB_U_CPDMASS, "ComputeCPDMass"},
    {FB_U_LABEL, "LabelAdvection"}, {FB_U_IMPOSEDDENSITY, "ImposedDensity"},
    {FB_U_ADDM, "AddM1/AddM2/AddM1toM10"}, {FB_U_CAVITY, "viscosity/density cavity"},
    {FB_U_TRANSITION, "aspect-ratio transition"}, {FB_U_LAMBDADOUBLING, "LambdaDoubling"},
    {FB_U_RELEASE, "planet ReleaseDate drift"}, {FB_U_FORCEDINNER, "ForcedInnerCircular"},
    {FB_U_RADIIFILE, "radii.dat"}, {FB_U_VISCRELEASE, "ReleaseDateViscosity"},
    {FB_U_DUSTTIMESTEP, "DustTimeStep-limited stepping"}, {FB_U_PARTICLES, "Lagrangian dust particles"},
    {FB_U_ADDNOISE, "AddNoise (wall-clock seeded)"}, {FB_U_PLANETACCRETION, "planet accretion"},
    {FB_U_FEELDISK, "planets feeling the disc"}, {FB_U_BINARY, "binary planets"},
    {FB_U_FEELOTHERS_FC, "FeelOthers with ForcedCircular"},
    {FB_U_ZZINTEGRATOR, "ZZIntegrator"},
    {FB_U_DUSTGROWTH, "DustGrowth"}, {FB_U_HILLREMOVAL, "RemoveDustFromPlanetsHillRadius"},
    {FB_U_INTERPOLATION, "NGP/CIC particle interpolation"}, {FB_U_DUSTSGZERO, "DustFeelSG Z"},
    {FB_U_SOFTWRITING, "SoftWriting with particles and self-gravity"},
  };
  size_t k;
  if (!p) return "";
  for (k = 0; k < sizeof names / sizeof names[0]; k++)
    if (p->unsupported & names[k].bit) return names[k].name;
  return "";
}

/* ------------------------------------------------------------- planets */
/* InitPlanetarySystem (src/Psys.c:96-203) for non-binary planets. */
int fb_planets_read_cfg(const fb_params *p, const char *path, fb_planets *out)
{
  FILE *input;
  char s[512], nm[512], test1[512], test2[512], test3[512], *s1;
  float mass, dist, accret;
  int i = 0;
  double massinvelocity;
  if (!p || !path || !out) return FB_ERR_INVALID;
  memset(out, 0, sizeof *out);
  input = fopen(path, "r");
  if (!input) return FB_ERR_IO;
  test1[0] = test2[0] = test3[0] = 0;
  while (fgets(s, 510, input) != NULL) {
    nm[0] = 0;
    sscanf(s, "%511s ", nm);
    if (isalpha((unsigned char)s[0])) {
      int feeldis = 1, feelothers = 1, binary = 0;
      if (i >= FB_MAX_PLANETS) { fclose(input); return FB_ERR_UNSUPPORTED; }
      s1 = s + strlen(nm);
      sscanf(s1 + strspn(s1, "\t :=>_"), "%f %f %f %511s %511s %511s", &dist, &mass, &accret,
             test1, test2, test3);
      out->mass[i] = (double)mass;
      out->initial_mass[i] = 0.0;
      out->final_mass[i] = out->mass[i];
      massinvelocity = (p->masstaper > 1e-3) ? 0.0 : out->final_mass[i];
      if (tolower((unsigned char)*test1) == 'n') feeldis = 0;
      if (tolower((unsigned char)*test2) == 'n') feelothers = 0;
      if (feeldis && p->forced_circular) { fclose(input); return FB_ERR_INVALID; }
      if (feelothers && p->forced_circular) { fclose(input); return FB_ERR_INVALID; }
      if (tolower((unsigned char)*test3) == 'y') binary = 1;
      out->x[i] = (double)dist * (1.0 + p->eccentricity);
      out->y[i] = 0.0;
      out->vy[i] = (double)sqrt(FB_G * (1.0 + massinvelocity) / dist) *
                   sqrt((1.0 - p->eccentricity) / (1.0 + p->eccentricity));
      out->vx[i] = -0.0000000001 * out->vy[i];
      out->acc[i] = accret;
      out->feeldisk[i] = feeldis;
      out->feelothers[i] = feelothers;
      out->binary[i] = binary;
      i++;
    }
  }
  fclose(input);
  out->nb = i;
  return FB_OK;
}

/* ------------------------------------------------------------- geometry */
int fb_geom_fill(const fb_params *p, const double *radii, fb_geom *g)
{
  int i, j, nr = p->nrad, ns = p->nsec;
  double drrsep;
  memset(g, 0, sizeof *g);
  g->nr = nr;
  g->ns = ns;
  g->radii = (double *)calloc(nr + 1, sizeof(double));
  g->rinf = (double *)calloc(nr + 1, sizeof(double));
  g->rsup = (double *)calloc(nr, sizeof(double));
  g->rmed = (double *)calloc(nr + 1, sizeof(double));
  g->surf = (double *)calloc(nr, sizeof(double));
  g->invrmed = (double *)calloc(nr, sizeof(double));
  g->invsurf = (double *)calloc(nr, sizeof(double));
  g->invdiffrsup = (double *)calloc(nr, sizeof(double));
  g->invrinf = (double *)calloc(nr, sizeof(double));
  g->invdiffrmed = (double *)calloc(nr + 1, sizeof(double));
  g->azimuth = (double *)calloc(ns, sizeof(double));
  g->cosaz = (double *)calloc(ns, sizeof(double));
  g->sinaz = (double *)calloc(ns, sizeof(double));
  if (!g->radii || !g->rinf || !g->rsup || !g->rmed || !g->surf || !g->invrmed ||
      !g->invsurf || !g->invdiffrsup || !g->invrinf || !g->invdiffrmed || !g->azimuth ||
      !g->cosaz || !g->sinaz) {
    fb_geom_free(g);
    return FB_ERR_NOMEM;
  }
  /* FillPolar1DArrays, src/SourceEuler.c:80-123 */
  drrsep = (p->rmax - p->rmin) / (double)nr;
  if (radii) {
    for (i = 0; i <= nr; i++) g->radii[i] = radii[i];
  } else if (p->log_grid) {
    for (i = 0; i <= nr; i++)
      g->radii[i] = p->rmin * exp((double)i / (double)nr * log(p->rmax / p->rmin));
  } else {
    for (i = 0; i <= nr; i++) g->radii[i] = p->rmin + drrsep * (double)(i);
  }
  for (i = 0; i < nr; i++) {
    g->rinf[i] = g->radii[i];
    g->rsup[i] = g->radii[i + 1];
    g->rmed[i] = 2.0 / 3.0 * (g->rsup[i] * g->rsup[i] * g->rsup[i] - g->rinf[i] * g->rinf[i] * g->rinf[i]);
    g->rmed[i] = g->rmed[i] / (g->rsup[i] * g->rsup[i] - g->rinf[i] * g->rinf[i]);
    g->surf[i] = 0.5 * (p->pmax - p->pmin) * (g->rsup[i] * g->rsup[i] - g->rinf[i] * g->rinf[i]) / (double)ns;
    g->invrmed[i] = 1.0 / g->rmed[i];
    g->invsurf[i] = 1.0 / g->surf[i];
    g->invdiffrsup[i] = 1.0 / (g->rsup[i] - g->rinf[i]);
    g->invrinf[i] = 1.0 / g->rinf[i];
  }
  g->rinf[nr] = g->radii[nr];
  for (i = 1; i < nr; i++) g->invdiffrmed[i] = 1.0 / (g->rmed[i] - g->rmed[i - 1]);
  /* src/SourceEuler.c:165-176 */
  for (j = 0; j < ns; j++) {
    g->azimuth[j] = p->pmin + (p->pmax - p->pmin) * (double)j / (double)ns;
    g->cosaz[j] = cos(g->azimuth[j]);
    g->sinaz[j] = sin(g->azimuth[j]);
  }
  return FB_OK;
}

void fb_geom_free(fb_geom *g)
{
  if (!g) return;
  free(g->radii); free(g->rinf); free(g->rsup); free(g->rmed); free(g->surf);
  free(g->invrmed); free(g->invsurf); free(g->invdiffrsup); free(g->invrinf);
  free(g->invdiffrmed); free(g->azimuth); free(g->cosaz); free(g->sinaz);
  memset(g, 0, sizeof *g);
}

/* ------------------------------------------------ reference profiles */
/* AspectRatio, src/Viscosity.c:107-123 (PhysicalTime = PhysicalTimeInitial
   and LAMBDADOUBLING = 0, TRANSITION* at their defaults: checked by the
   parser). */
double fb_host_aspect_ratio(const fb_params *p, double rad)
{
  double aspectratio = p->aspectratio;
  double rmin = 0.0 - 1.0 * p->aspectratio;
  double rmax = 0.0 + 1.0 * p->aspectratio;
  if ((rad >= rmin) && (rad <= rmax)) aspectratio *= exp((rmax - rad) / (rmax - rmin) * log(1.0));
  return aspectratio;
}

/* Sigma, src/Theo.c:13-60 with no cavity and ScalingFactor = 1 */
double fb_host_sigma(const fb_params *p, double r)
{
  double cavity = 1.0, scaling = 1.0;
  return cavity * scaling * p->sigma0 * pow(r, -p->sigmaslope);
}

/* Energy, src/Theo.c:156-170 */
double fb_host_energy(const fb_params *p, double r)
{
  double cavity = 1.0, scaling = 1.0;
  double energy0 = 1.0 / 1.0 / (p->adiabaticindex - 1.0) * fb_host_sigma(p, r) *
                   pow(p->aspectratio, 2.0) * pow(r, -1.0 + 2.0 * p->flaringindex);
  return cavity * scaling * energy0;
}

/* compute_smoothing, src/Force.c:255-263 */
double fb_host_smoothing(const fb_params *p, double r)
{
  return p->thicknesssmoothing * fb_host_aspect_ratio(p, r) * pow(r, 1.0 + p->flaringindex);
}

/* ------------------------------------------------- initial conditions */
int fb_init_state(const fb_params *p, fb_ctx *ctx, double noise_amp, long noise_seed,
                  fb_state *st, fb_profiles *prof)
{
  fb_geom gl, *g;
  const fb_geom *gc = ctx ? fb_ctx_geom(ctx) : NULL;
  int i, j, nr, ns, rc, k;
  size_t nf;
  double *cs = NULL, *axisg = NULL;
  if (!p || !st || !prof || !st->dens || !st->vrad || !st->vtheta || !st->energy)
    return FB_ERR_INVALID;
  if (!prof->sigma_med || !prof->sigma_inf || !prof->energy_med || !prof->vtheta_med ||
      !prof->vrad_med || !prof->global_soundspeed)
    return FB_ERR_INVALID;
  if (p->self_gravity && !ctx) return FB_ERR_INVALID;
  nr = p->nrad;
  ns = p->nsec;
  nf = (size_t)(nr + 1) * ns;
  if (gc) {
    g = (fb_geom *)gc;
  } else {
    rc = fb_geom_fill(p, NULL, &gl);
    if (rc) return rc;
    g = &gl;
  }
  memset(st->dens, 0, nf * sizeof(double));
  memset(st->vrad, 0, nf * sizeof(double));
  memset(st->vtheta, 0, nf * sizeof(double));
  memset(st->energy, 0, nf * sizeof(double));
  for (i = 0; i < nr; i++) {
    prof->energy_med[i] = 0.0;
    prof->global_soundspeed[i] = 0.0;
  }
  rc = fb_planets_read_cfg(p, p->planetconfig, &st->planets);
  if (rc) goto done;

  /* InitGasDensity (src/Pframeforce.c:297-339), FillSigma (Theo.c:89) */
  for (i = 0; i < nr; i++) {
    prof->sigma_med[i] = fb_host_sigma(p, g->rmed[i]);
    prof->sigma_inf[i] = fb_host_sigma(p, g->rinf[i]);
  }
  for (i = 0; i < nr; i++)
    for (j = 0; j < ns; j++) st->dens[j + i * ns] = prof->sigma_med[i];
  if (p->add_noise) {
    /* AddNoise (Pframeforce.c:317-320): 1e-3 relative, drand48 from the seed */
    fb_rand48 r48;
    fb_srand48(&r48, noise_seed);
    for (i = 0; i < nr; i++)
      for (j = 0; j < ns; j++)
        st->dens[j + i * ns] += 1e-3 * prof->sigma_med[i] * (2.0 * fb_drand48(&r48) - 1.0);
  }
  if (noise_amp != 0.0) {
    fb_rand48 r48;
    fb_srand48(&r48, noise_seed);
    for (i = 0; i < nr; i++)
      for (j = 0; j < ns; j++)
        st->dens[j + i * ns] += noise_amp * prof->sigma_med[i] * (2.0 * fb_drand48(&r48) - 1.0);
  }
  /* InitGasEnergy (src/Pframeforce.c:422-439) */
  if (p->energy_equation) {
    for (i = 0; i < nr; i++) prof->energy_med[i] = fb_host_energy(p, g->rmed[i]);
    for (i = 0; i < nr; i++)
      for (j = 0; j < ns; j++) st->energy[j + i * ns] = prof->energy_med[i];
  }
  /* Self-gravity at t=0 (main.c:176-186): SG acceleration of the initial
     density, then init_planetarysys_withSG (src/sgsysinit.c:3-49). */
  if (p->self_gravity) {
    axisg = (double *)calloc(nr, sizeof(double));
    if (!axisg) { rc = FB_ERR_NOMEM; goto done; }
    rc = fb_sg_axisym_accel(ctx, st->dens, axisg);
    if (rc) goto done;
    for (k = 0; k < st->planets.nb; k++) {
      double x = st->planets.x[k], y = st->planets.y[k];
      double r = sqrt(x * x + y * y);
      double dist = (double)(r / (1. + p->eccentricity));
      double sgacc;
      if (dist < g->rmed[nr - 1]) {
        int ipl = 0;
        double ri, rip1, dr;
        while ((g->rmed[ipl] <= dist) && (ipl < nr - 2)) ipl++;
        ri = g->rmed[ipl];
        rip1 = g->rmed[ipl + 1];
        dr = rip1 - ri;
        sgacc = (dist - ri) * axisg[ipl + 1] + (rip1 - dist) * axisg[ipl];
        sgacc /= dr;
      } else {
        sgacc = axisg[nr - 1];
      }
      st->planets.vy[k] *= (double)sqrt(1. - dist * dist * sgacc / FB_G / (1.0 + st->planets.mass[k]));
    }
  }
  st->omega_frame = p->omegaframe;
  if (p->corotating && st->planets.nb > 0) {
    /* main.c:228-247: the first planet's angular frequency, from its orbit
       (GetPsysInfo FREQUENCY, Psys.c:281-297) or, with self-gravity, v / r */
    const double x = st->planets.x[0], y = st->planets.y[0];
    const double vx = st->planets.vx[0], vy = st->planets.vy[0];
    if (!p->self_gravity) {
      const double m = st->planets.mass[0] + 1.;
      const double h = x * vy - y * vx;
      const double d = sqrt(x * x + y * y);
      const double Ax = x * vy * vy - y * vx * vy - FB_G * m * x / d;
      const double Ay = y * vx * vx - x * vx * vy - FB_G * m * y / d;
      const double e = sqrt(Ax * Ax + Ay * Ay) / m;
      const double a = h * h / FB_G / m / (1. - e * e);
      st->omega_frame = sqrt(m / a / a / a);
    } else {
      const double r = sqrt(x * x + y * y), v = sqrt(vx * vx + vy * vy);
      st->omega_frame = v / r;
    }
  }

  /* InitEuler: ComputeSoundSpeed (src/SourceEuler.c:2323-2343) */
  cs = (double *)calloc(nf, sizeof(double));
  if (!cs) { rc = FB_ERR_NOMEM; goto done; }
  for (i = 0; i < nr; i++) {
    double cs_buf = 0.0;
    if (!p->energy_equation)
      cs_buf = fb_host_aspect_ratio(p, g->rmed[i]) * sqrt(FB_G * 1.0 / g->rmed[i]) *
               pow(g->rmed[i], p->flaringindex);
    for (j = 0; j < ns; j++) {
      size_t l = (size_t)i * ns + j;
      if (!p->energy_equation)
        cs[l] = cs_buf;
      else
        cs[l] = sqrt(p->adiabaticindex * (p->adiabaticindex - 1.0) * st->energy[l] / st->dens[l]);
    }
  }
  /* InitGasVelocities, src/Pframeforce.c:442-641, no centrifugal balance */
  for (i = 0; i < nr; i++) {
    double r = g->rmed[i];
    double omega = sqrt(FB_G * 1.0 / r / r / r);
    double myvtheta = omega * r *
                      sqrt(1.0 - pow(p->aspectratio, 2.0) * pow(r, 2.0 * p->flaringindex) *
                                     (1. + p->sigmaslope - 2.0 * p->flaringindex));
    for (j = 0; j < ns; j++) st->vtheta[j + i * ns] = myvtheta;
  }
  if (p->self_gravity) {
    /* loop runs to i <= nr with Rmed[nr] = 0 (a global never set) */
    for (i = 0; i <= nr; i++) {
      double r = (i < nr) ? g->rmed[i] : 0.0;
      double a = (i < nr) ? axisg[i] : 0.0;
      for (j = 0; j < ns; j++) {
        size_t l = (size_t)i * ns + j;
        double vt2 = st->vtheta[l] * st->vtheta[l];
        vt2 -= r * a;
        st->vtheta[l] = sqrt(vt2);
      }
    }
  }
  for (i = 0; i < nr; i++) {
    double r = g->rmed[i];
    for (j = 0; j < ns; j++) st->vtheta[(size_t)i * ns + j] -= st->omega_frame * r;
  }
  if (p->alphaviscosity != 0.0) {
    /* mpi_make1Dprofile (src/axilib.c:5-60), one process */
    for (i = 0; i < nr; i++) {
      double acc = 0.0;
      for (j = 0; j < ns; j++) acc += cs[(size_t)i * ns + j];
      acc /= (double)ns;
      prof->global_soundspeed[i] = acc;
    }
  }
  for (i = 0; i < nr; i++) {
    double r = g->rmed[i], ri = g->rinf[i], viscosity;
    if (p->alphaviscosity != 0.0 || p->viscosity != 0.0) {
      /* FViscosity (src/Viscosity.c:23-69) at r = Rmed[i] */
      if (p->alphaviscosity != 0.0)
        viscosity = p->alphaviscosity * prof->global_soundspeed[i] * prof->global_soundspeed[i] *
                    pow(r, 1.5);
      else
        viscosity = p->viscosity;
    } else {
      viscosity = 0.0;
    }
    for (j = 0; j < ns; j++) {
      size_t l = (size_t)i * ns + j;
      if (p->imposeddiskdrift != 0.0)
        st->vrad[l] = p->imposeddiskdrift * p->sigma0 / prof->sigma_inf[i] / ri;
      else if (p->alphaviscosity != 0.0)
        st->vrad[l] -= 3.0 * viscosity / r * (-p->sigmaslope + 2.0 * p->flaringindex + 1.0);
      else
        st->vrad[l] -= 3.0 * viscosity / r * (-p->sigmaslope + .5);
    }
  }
  for (i = 0; i < nr; i++) {
    prof->vtheta_med[i] = st->vtheta[(size_t)i * ns] + g->rmed[i] * st->omega_frame;
    prof->vrad_med[i] = st->vrad[(size_t)i * ns];
  }
  st->physical_time = 0.0;
  st->physical_time_initial = 0.0;
  st->lost_mass = 0.0;
  st->mindt = p->mindt;
  st->maxdt = p->maxdt;
  for (k = 0; k < 3; k++) {
    st->stardiscbarycenter_x[k] = 0.0;
    st->stardiscbarycenter_y[k] = 0.0;
  }
  rc = FB_OK;
done:
  free(cs);
  free(axisg);
  if (!gc) fb_geom_free(&gl);
  return rc;
}

/* ComputeCodeUnits (src/LowTasks.c:202-213) */
double fb_unit_length(const fb_params *p) { return 1.49598e11 * p->factorunitlength; }
double fb_unit_mass(const fb_params *p) { return 1.9891e30 * p->factorunitmass; }
double fb_unit_time(const fb_params *p)
{
  return sqrt(pow(fb_unit_length(p), 3.) / 6.673e-11 / fb_unit_mass(p));
}
double fb_unit_temperature(const fb_params *p)
{
  const double mmw = 2.35 * p->factormmw;
  return mmw * 8.0841643e-15 * fb_unit_mass(p) / fb_unit_length(p);
}

/* InitDustSystem (src/Dsys.c:128-262), new particles, one process. */
int fb_init_dust(const fb_params *p, fb_ctx *ctx, long seed, fb_dust_state *st)
{
  fb_geom gl, *g;
  const fb_geom *gc = ctx ? fb_ctx_geom(ctx) : NULL;
  fb_rand48 r48;
  double C1, C2, rmindust, rmaxdust, aziinf0, azisupl, unit_length;
  double *axisg = NULL;
  int i, n, rc;
  if (!p || !st || !st->r || !st->th || !st->vr || !st->vth || !st->l || !st->size || !st->stokes)
    return FB_ERR_INVALID;
  n = p->nbpart;
  if (n <= 0 || st->n != n) return FB_ERR_INVALID;
  if (p->self_gravity && !ctx) return FB_ERR_INVALID;
  if (p->sizeminpart == p->sizemaxpart && p->sizepartslope != 0.0) return FB_ERR_INVALID;  /* Dsys.c:151-155 */
  if (gc) {
    g = (fb_geom *)gc;
  } else {
    rc = fb_geom_fill(p, NULL, &gl);
    if (rc) return rc;
    g = &gl;
  }
  unit_length = fb_unit_length(p);
  rmindust = (p->rmindust == 0.0) ? p->rmin : p->rmindust;
  rmaxdust = (p->rmaxdust == 0.0) ? p->rmax : p->rmaxdust;
  /* AziInf[0], AziSup[NSEC-1] (src/SourceEuler.c:176-179) */
  aziinf0 = g->azimuth[0] - 0.5 * (p->pmax - p->pmin) / (double)p->nsec;
  azisupl = g->azimuth[p->nsec - 1] + 0.5 * (p->pmax - p->pmin) / (double)p->nsec;
  fb_srand48(&r48, seed);
  if (p->sizeminpart != p->sizemaxpart) {
    if (p->sizepartslope != 1.0) {
      C1 = pow(p->sizemaxpart, 1.0 - p->sizepartslope);
      C2 = pow(p->sizeminpart, 1.0 - p->sizepartslope);
      for (i = 0; i < n; i++)
        st->size[i] = pow(C2 + (C1 - C2) * fb_drand48(&r48), 1.0 / (1.0 - p->sizepartslope)) / unit_length;
    } else {
      for (i = 0; i < n; i++)
        st->size[i] = p->sizeminpart * exp(fb_drand48(&r48) * log(p->sizemaxpart / p->sizeminpart)) / unit_length;
    }
  } else {
    for (i = 0; i < n; i++) st->size[i] = p->sizeminpart / unit_length;
  }
  if (p->dustslope != 1.0) {
    C1 = pow(rmaxdust, 1.0 - p->dustslope);
    C2 = pow(rmindust, 1.0 - p->dustslope);
    for (i = 0; i < n; i++) st->r[i] = pow(C2 + (C1 - C2) * fb_drand48(&r48), 1.0 / (1.0 - p->dustslope));
  } else {
    for (i = 0; i < n; i++) st->r[i] = rmindust * exp(fb_drand48(&r48) * log(rmaxdust / rmindust));
  }
  for (i = 0; i < n; i++) st->th[i] = aziinf0 + fb_drand48(&r48) * (azisupl - aziinf0);
  if (p->self_gravity) {
    axisg = (double *)calloc(p->nrad, sizeof(double));
    if (!axisg) { rc = FB_ERR_NOMEM; goto done; }
    rc = fb_sg_axisym_accel_device(ctx, axisg);
    if (rc) goto done;
  }
  for (i = 0; i < n; i++) {
    st->vr[i] = 0.0;
    st->stokes[i] = 0.0;
    if (!p->self_gravity) {
      st->vth[i] = pow(st->r[i], -0.5);
    } else {
      double dist = st->r[i], ri, rip1, dr, sgacc;
      int ipl = 0;
      while ((g->rmed[ipl] <= dist) && (ipl < p->nrad - 2)) ipl++;
      ri = g->rmed[ipl];
      rip1 = g->rmed[ipl + 1];
      dr = rip1 - ri;
      sgacc = (dist - ri) * axisg[ipl + 1] + (rip1 - dist) * axisg[ipl];
      sgacc /= dr;
      st->vth[i] = pow(st->r[i], -0.5) * sqrt(1.0 - dist * dist * sgacc);
    }
    st->l[i] = st->r[i] * st->vth[i];
  }
  st->rng_x = r48.x;
  st->kicks = 0;
  st->carry[0] = st->carry[1] = 0.0;
  /* Particles_Mass: the dust surface density is only initialised with a
     dust fluid, so it is zero here (main.c:167-200) */
  st->particles_mass = 0.0;
  rc = FB_OK;
done:
  free(axisg);
  if (!gc) fb_geom_free(&gl);
  return rc;
}

int fb_struct_size(int which)
{
  switch (which) {
    case 0: return (int)sizeof(fb_params);
    case 1: return (int)sizeof(fb_planets);
    case 2: return (int)sizeof(fb_state);
    case 3: return (int)sizeof(fb_profiles);
    case 4: return (int)sizeof(fb_step_report);
    case 5: return (int)sizeof(fb_dust_state);
    case 6: return (int)sizeof(fb_tuning);
    default: return -1;
  }
}
