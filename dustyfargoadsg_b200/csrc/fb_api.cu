// fb_api.cu -- the C ABI of libfargo_b200.so: device context, upload /
// download, and the substep sequence of AlgoGas (src/SourceEuler.c:326-719).
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include "fb_dev.cuh"

#define FB_PROFILE_POINTS 64
enum {
  ST_CFL, ST_SUB0, ST_CONTROL, ST_SOUND, ST_POT, ST_SUB1, ST_SG, ST_SGCOLS, ST_SGINV, ST_SGUPD,
  ST_VTERMS, ST_VUPDATE,
  ST_SUB2, ST_EVTERMS, ST_SUB3, ST_TRAD, ST_TAZI, ST_TVR, ST_DAMP, ST_DUST, ST_TVMED, FB_NSTAGE
};
static const char *stage_names[FB_NSTAGE] = {
  "cfl_forces", "substep0", "controller", "soundspeed", "potential", "substep1", "sg_rows_fwd",
  "sg_cols", "sg_rows_inv", "sg_update",
  "viscous_terms", "viscous_update", "substep2", "energy_viscous_terms", "substep3",
  "transport_radial", "transport_azimuthal", "transport_vr_boundary", "damping", "dust_particles",
  "transport_ring_means"};

struct fb_ctx {
  fb_params p;
  fb_geom g;
  int nr, ns;
  size_t nf;
  cudaStream_t st;
  cudaEvent_t ev0, ev1;
  cudaStream_t st_planets;            // branch of the planets' step (k_planets)
  cudaEvent_t ev_fork, ev_planets;    // its start and end within a substep
  cudaStream_t st_sg;                 // branch of the self-gravity convolution
  cudaEvent_t ev_sg_fork, ev_sg_done;
  cudaEvent_t ev_vm_fork, ev_vm_done;  // the tile variant's ring means, on the SG stream beside SubStep3 / radial
  KP k;
  std::vector<void *> allocs;
  fb_ctl *d_ctl;
  fb_ctl *h_ctl;  // pinned mirror
  double *d_diag;
  double *h_diag; // pinned
  fb_sg *sg;
  int uploaded;
  char err[512];
  // host copies of the tables that depend on uploaded profiles
  std::vector<double> h_supp;
  // launch accounting and optional per-stage profiling
  long long launches;
  int profiling;
  std::vector<cudaEvent_t> pev;   // one per recorded point of a substep
  std::vector<int> pseq;          // stage id of each recorded interval
  double pms[FB_NSTAGE];
  long long pcount[FB_NSTAGE];
  // one DT as a CUDA graph: a conditional WHILE node around the substep
  cudaGraph_t gdt;
  cudaGraphExec_t gdt_exec;
  int graph_state;            // 0 not built, 1 ready, -1 unavailable
  long long launches_per_substep;
  int substep_cap;
  // Lagrangian particles (nbpart > 0)
  PP pp;
  int has_dust, dust_uploaded;
  fb_dust_ctl *h_dc;  // pinned mirror of pp.dc
};

static void set_err(fb_ctx *c, const char *fmt, ...)
{
  if (!c) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(c->err, sizeof c->err, fmt, ap);
  va_end(ap);
}

#define CK(call)                                                                    \
  do {                                                                              \
    cudaError_t _e = (call);                                                        \
    if (_e != cudaSuccess) {                                                        \
      set_err(ctx, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e)); \
      return FB_ERR_CUDA;                                                           \
    }                                                                               \
  } while (0)

static double *dalloc(fb_ctx *ctx, size_t n)
{
  void *p = NULL;
  if (cudaMalloc(&p, n * sizeof(double)) != cudaSuccess) return NULL;
  cudaMemset(p, 0, n * sizeof(double));
  ctx->allocs.push_back(p);
  return (double *)p;
}

static const double *dtable(fb_ctx *ctx, const double *h, size_t n)
{
  double *d = dalloc(ctx, n);
  if (d && h) cudaMemcpy(d, h, n * sizeof(double), cudaMemcpyHostToDevice);
  return d;
}

extern "C" int fb_select_device(int device)
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) return FB_ERR_NODEVICE;
  if (device < 0 || device >= n) return FB_ERR_INVALID;
  return cudaSetDevice(device) == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

extern "C" const fb_geom *fb_ctx_geom(const fb_ctx *ctx) { return ctx ? &ctx->g : NULL; }
const KP *fb_ctx_kp(const fb_ctx *ctx) { return ctx ? &ctx->k : NULL; }
KP *fb_ctx_kp_mut(fb_ctx *ctx) { return ctx ? &ctx->k : NULL; }
cudaStream_t fb_ctx_stream(const fb_ctx *ctx) { return ctx ? ctx->st : NULL; }
void fb_ctx_count_launches(fb_ctx *ctx, int n) { if (ctx) ctx->launches += n; }

extern "C" const char *fb_strerror(int code)
{
  switch (code) {
    case FB_OK: return "ok";
    case FB_ERR_INVALID: return "invalid argument or parameter";
    case FB_ERR_UNSUPPORTED: return "feature not supported by this build";
    case FB_ERR_CUDA: return "CUDA error";
    case FB_ERR_NOMEM: return "out of memory";
    case FB_ERR_NAN: return "non-finite value in the gas state";
    case FB_ERR_NEGATIVE: return "negative density or energy";
    case FB_ERR_SUBSTEPS: return "CFL substep count out of range";
    case FB_ERR_TIMEOUT: return "bounded device wait timed out";
    case FB_ERR_IO: return "I/O error";
    case FB_ERR_STATE: return "call made in the wrong order";
    case FB_ERR_NODEVICE: return "no CUDA device";
    default: return "unknown error";
  }
}

extern "C" const char *fb_last_error(const fb_ctx *ctx) { return ctx ? ctx->err : "no context"; }

extern "C" const char *fb_build_info(void)
{
#if FB_FAST
  return "libfargo_b200_fast sm_100a fp64 --fmad=true approximate-reciprocal slopes abi 2";
#else
  return "libfargo_b200 sm_100a fp64 --fmad=false abi 2";
#endif
}

// Particle arrays, the grids the gas step leaves for them, and the constants
// of the particle update (Dsys.c:308-331).
static int dust_create(fb_ctx *ctx)
{
  const fb_params *p = &ctx->p;
  KP &k = ctx->k;
  PP &pp = ctx->pp;
  const int n = p->nbpart, ns = ctx->ns;
  const size_t nf = ctx->nf;
  if (p->omegaframe != 0.0) {
    set_err(ctx, "particles need a non-rotating frame (OMEGAFRAME = 0)");
    return FB_ERR_UNSUPPORTED;
  }
  double **grids[] = {&k.indpot, &k.rgp, &k.agp, &k.rind, &k.aind, &k.rsga, &k.asga};
  for (size_t f = 0; f < sizeof grids / sizeof grids[0]; f++)
    if (!(*grids[f] = dalloc(ctx, nf))) return FB_ERR_NOMEM;
  k.particles = 1;
  k.dust_feel_planets = p->dust_feel_planets;
  k.dust_feel_disk = p->dust_feel_disk;
  memset(&pp, 0, sizeof pp);
  pp.n = n;
  // candidate uniform pairs per substep: accepted ones (rate pi/4) must cover
  // one Gaussian pair per kicked particle plus the odd one
  pp.ncand = (int)((long long)(n + 4) * 27 / 20 + 2048 + 256);
  double **arrays[] = {&pp.r, &pp.th, &pp.vr, &pp.vth, &pp.l, &pp.size, &pp.st};
  for (size_t f = 0; f < sizeof arrays / sizeof arrays[0]; f++)
    if (!(*arrays[f] = dalloc(ctx, n))) return FB_ERR_NOMEM;
  const int nsb = (n + 1023) / 1024, ncb = (pp.ncand + 255) / 256;
  pp.ncells = ctx->nr * ctx->ns + 1;
  int **ints[] = {&pp.flag, &pp.kidx, &pp.kick_bsum, &pp.cand_flag, &pp.cand_bsum,
                  &pp.perm, &pp.key, &pp.cell_count, &pp.cell_bsum, &pp.orig, &pp.oscratch};
  const size_t isz[] = {(size_t)n, (size_t)n, (size_t)nsb, (size_t)pp.ncand, (size_t)ncb,
                        (size_t)n, (size_t)n, (size_t)pp.ncells, (size_t)(pp.ncells + 1023) / 1024,
                        (size_t)n, (size_t)n};
  for (size_t f = 0; f < 11; f++) {
    void *d = NULL;
    if (cudaMalloc(&d, isz[f] * sizeof(int)) != cudaSuccess) return FB_ERR_NOMEM;
    cudaMemset(d, 0, isz[f] * sizeof(int));
    ctx->allocs.push_back(d);
    *ints[f] = (int *)d;
  }
  {
    void *d = NULL;
    if (cudaMalloc(&d, ((size_t)n + 4) * sizeof(double2)) != cudaSuccess) return FB_ERR_NOMEM;
    ctx->allocs.push_back(d);
    pp.pairs = (double2 *)d;
    if (cudaMalloc(&d, sizeof(fb_dust_ctl)) != cudaSuccess) return FB_ERR_NOMEM;
    cudaMemset(d, 0, sizeof(fb_dust_ctl));
    ctx->allocs.push_back(d);
    pp.dc = (fb_dust_ctl *)d;
    if (cudaMallocHost((void **)&ctx->h_dc, sizeof(fb_dust_ctl)) != cudaSuccess) return FB_ERR_NOMEM;
    memset(ctx->h_dc, 0, sizeof(fb_dust_ctl));
  }
  // azimuths of the cell centres and interfaces (SourceEuler.c:162-174)
  const fb_geom &g = ctx->g;
  const double half = 0.5 * (p->pmax - p->pmin) / (double)ns;
  std::vector<double> aziinf(ns);
  for (int j = 0; j < ns; j++) aziinf[j] = g.azimuth[j] - half;
  pp.azimuth = dtable(ctx, g.azimuth, ns);
  pp.aziinf = dtable(ctx, aziinf.data(), ns);
  pp.aziinf0 = aziinf[0];
  pp.azisupl = g.azimuth[ns - 1] + half;
  pp.delta_r = p->log_grid ? log(g.rsup[0] / g.rinf[0]) : g.rsup[0] - g.rinf[0];
  pp.delta_phi = (g.azimuth[0] + half) - (g.azimuth[0] - half);
  pp.rmin = p->rmin;
  pp.rmax = p->rmax;
  const double unit_length = fb_unit_length(p), unit_mass = fb_unit_mass(p);
  pp.unit_mass = unit_mass;
  pp.inv_unit_length2 = pow(unit_length, -2.0);
  pp.dust_density_cu = p->rhopart * 1000.0 * pow(unit_length, 3.) / unit_mass;
  pp.aspectratio = p->aspectratio;
  pp.thicksmoothing = p->thicknesssmoothing;
  pp.flaringindex = p->flaringindex;
  pp.log_grid = p->log_grid;
  pp.feel_disk = p->dust_feel_disk;
  pp.feel_planets = p->dust_feel_planets;
  pp.feel_sg = p->dust_feel_sg;
  pp.feel_turb = p->dust_feel_turb;
  pp.sfta = p->sfta;
  pp.restokes = p->write_dust_density;
  // DUSTFEEDBACK with the particle mass of a run without a dust fluid (zero,
  // main.c:187-201): the feedback accelerations and heating are exact zeros
  // and only the stopping-time bound on the substep remains
  if (p->dust_feedback) k.dust_min_ts = &pp.dc->min_ts;
  if (!pp.azimuth || !pp.aziinf) return FB_ERR_NOMEM;
  if (!(pp.pscratch = dalloc(ctx, 7 * (size_t)n))) return FB_ERR_NOMEM;
  // first guess of a radius's ring: the grid law of the radii
  pp.ring_r0 = g.rinf[0];
  pp.ring_inv_r0 = 1.0 / g.rinf[0];
  pp.ring_inv_step = p->log_grid ? (double)ctx->nr / log(g.rsup[ctx->nr - 1] / g.rinf[0])
                                 : (double)ctx->nr / (g.rsup[ctx->nr - 1] - g.rinf[0]);
  {
    std::vector<double> lri(ctx->nr + 1), lrm(ctx->nr);
    for (int i = 0; i <= ctx->nr; i++) lri[i] = log(g.rinf[i]);
    for (int i = 0; i < ctx->nr; i++) lrm[i] = log(g.rmed[i]);
    pp.log_rinf = dtable(ctx, lri.data(), ctx->nr + 1);
    pp.log_rmed = dtable(ctx, lrm.data(), ctx->nr);
    if (!pp.log_rinf || !pp.log_rmed) return FB_ERR_NOMEM;
  }
  ctx->has_dust = 1;
  return FB_OK;
}

// ------------------------------------------------------------------ create
extern "C" int fb_create(const fb_params *p, const double *radii, fb_ctx **out)
{
  if (!p || !out) return FB_ERR_INVALID;
  *out = NULL;
  if (p->unsupported) return FB_ERR_UNSUPPORTED;
  if (p->nrad < 4 || p->nsec < 2) return FB_ERR_INVALID;
  if ((p->open_inner || p->non_reflecting) && p->nrad < 8) return FB_ERR_INVALID;  // the edges span 4 rings each
  if (p->self_gravity && !p->log_grid) return FB_ERR_INVALID;  // sginit.c:6-7
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return FB_ERR_NODEVICE;
  fb_ctx *ctx = new fb_ctx();
  ctx->p = *p;
  ctx->nr = p->nrad;
  ctx->ns = p->nsec;
  ctx->nf = (size_t)(p->nrad + 1) * p->nsec;
  ctx->err[0] = 0;
  int rc = fb_geom_fill(p, radii, &ctx->g);
  if (rc) { delete ctx; return rc; }
  if (getenv("FB_NO_PDL")) fb_pdl = 0;  // launches without programmatic dependencies
  rc = fb_gas_prepare(ctx->ns, p->energy_equation);
  if (rc) { set_err(ctx, "ring of %d doubles does not fit in shared memory", ctx->ns); fb_geom_free(&ctx->g); delete ctx; return rc; }
  if (cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return FB_ERR_CUDA; }
  cudaEventCreate(&ctx->ev0);
  cudaEventCreate(&ctx->ev1);
  if (cudaStreamCreateWithFlags(&ctx->st_planets, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_planets, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->st_sg, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_sg_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_sg_done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_vm_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_vm_done, cudaEventDisableTiming) != cudaSuccess) {
    fb_destroy(ctx);
    return FB_ERR_CUDA;
  }
  const int nr = ctx->nr, ns = ctx->ns;
  const size_t nf = ctx->nf;
  KP &k = ctx->k;
  memset(&k, 0, sizeof k);
  k.nr = nr;
  k.ns = ns;
  k.nf = nf;
  double **fields[] = {&k.rho, &k.vr, &k.vt, &k.e, &k.cs, &k.pres, &k.pot, &k.vri, &k.vti,
                       &k.divv, &k.trr, &k.tpp, &k.trp, &k.vischeat, &k.q[0], &k.q[1], &k.q[2],
                       &k.q[3], &k.q[4], &k.q[5], &k.rho_t, &k.sg_accr, &k.sg_acct,
                       &k.azt_buf[0], &k.azt_buf[1], &k.azt_buf[2]};
  for (size_t f = 0; f < sizeof fields / sizeof fields[0]; f++) {
    *fields[f] = dalloc(ctx, nf);
    if (!*fields[f]) { fb_destroy(ctx); return FB_ERR_NOMEM; }
  }
  k.lost0 = dalloc(ctx, ns);
  k.azt_vmed = dalloc(ctx, nr);
  if (!k.lost0 || !k.azt_vmed) { fb_destroy(ctx); return FB_ERR_NOMEM; }
  if (p->energy_equation) {  // only the energy test can crash (DetectCrash as AlgoGas uses it)
    k.crash_snap = dalloc(ctx, (size_t)4 * nr * ns);
    if (!k.crash_snap) { fb_destroy(ctx); return FB_ERR_NOMEM; }
  }
  // 1-D tables (host, glibc libm; see fb_host.c)
  const fb_geom &g = ctx->g;
  std::vector<double> cs_ring(nr), p15(nr), dxrad(nr), dxth(nr), invdxth(nr), dxth_cfl(nr), mindx2(nr);
  std::vector<double> beta(nr), dlam(nr, 0.0), dtau(nr, 1.0);
  std::vector<int> drings;
  for (int i = 0; i < nr; i++) {
    const double r = g.rmed[i];
    cs_ring[i] = fb_host_aspect_ratio(p, r) * sqrt(FB_G * 1.0 / r) * pow(r, p->flaringindex);
    p15[i] = pow(r, 1.5);
    dxrad[i] = g.rsup[i] - g.rinf[i];
    dxth[i] = (p->pmax - p->pmin) / (double)ns * g.rmed[i];   // SourceEuler.c:928, TransportEuler.c:405
    invdxth[i] = 1.0 / dxth[i];
    dxth_cfl[i] = g.rmed[i] * (p->pmax - p->pmin) / (double)ns;  // SourceEuler.c:1344
    {
      double a = dxrad[i], b = dxth_cfl[i];
      double m = (b < a) ? b : a;
      mindx2[i] = pow(m, 2.0);
    }
    beta[i] = p->betacoolingtime * pow(r, -p->betacoolingslope);  // Theo.c:216-222
    if (p->evanescent && ((r < p->wkzrmin) || (r > p->wkzrmax))) {
      double damping = 0.0, T = 1.0;
      if (r < p->wkzrmin) {
        damping = (r - p->wkzrmin) / (g.rmed[0] - p->wkzrmin);
        T = p->dampingtodynamicaltimeratio * pow(r, 1.5);
      }
      if (r > p->wkzrmax) {
        damping = (r - p->wkzrmax) / (g.rmed[nr - 1] - p->wkzrmax);
        T = p->dampingtodynamicaltimeratio * pow(r, 1.5);
      }
      dlam[i] = damping * damping;
      dtau[i] = T;
      drings.push_back(i);
    }
  }
  k.rinf = dtable(ctx, g.rinf, nr + 1);
  k.rsup = dtable(ctx, g.rsup, nr);
  k.rmed = dtable(ctx, g.rmed, nr + 1);
  k.surf = dtable(ctx, g.surf, nr);
  k.invrmed = dtable(ctx, g.invrmed, nr);
  k.invsurf = dtable(ctx, g.invsurf, nr);
  k.invdiffrsup = dtable(ctx, g.invdiffrsup, nr);
  k.invrinf = dtable(ctx, g.invrinf, nr);
  k.invdiffrmed = dtable(ctx, g.invdiffrmed, nr + 1);
  k.cosaz = dtable(ctx, g.cosaz, ns);
  k.sinaz = dtable(ctx, g.sinaz, ns);
  k.cs_ring = dtable(ctx, cs_ring.data(), nr);
  k.gcs = dalloc(ctx, nr);
  k.p15 = dtable(ctx, p15.data(), nr);
  k.dxrad = dtable(ctx, dxrad.data(), nr);
  k.dxtheta = dtable(ctx, dxth.data(), nr);
  k.invdxtheta = dtable(ctx, invdxth.data(), nr);
  k.dxtheta_cfl = dtable(ctx, dxth_cfl.data(), nr);
  k.mindx2 = dtable(ctx, mindx2.data(), nr);
  k.supp_torque = dalloc(ctx, nr);
  k.sigmamed = dalloc(ctx, nr);
  k.energymed = dalloc(ctx, nr);
  k.vthetamed = dalloc(ctx, nr);
  k.vradmed = dalloc(ctx, nr);
  k.betatab = dtable(ctx, beta.data(), nr);
  k.damp_lam = dtable(ctx, dlam.data(), nr);
  k.damp_tau = dtable(ctx, dtau.data(), nr);
  {
    int *d = NULL;
    if (!drings.empty()) {
      cudaMalloc(&d, drings.size() * sizeof(int));
      cudaMemcpy(d, drings.data(), drings.size() * sizeof(int), cudaMemcpyHostToDevice);
      ctx->allocs.push_back(d);
    }
    k.damp_rings = d;
    k.n_damp_rings = (int)drings.size();
  }
  k.vh_l1 = log(g.rmed[0] / g.rmed[1]);
  k.vh_l2 = log(g.rmed[1] / g.rmed[2]);
  k.ringmin = dalloc(ctx, nr);
  k.vmoy = dalloc(ctx, nr);
  k.vt_part = dalloc(ctx, (size_t)nr * ((ns + 31) / 32));  // CTAs of >= 32 azimuths
  {
    // the CFL kernel leaves one set of force/mass partials per ring
    const int nb = nr;
    k.n_partial_blocks = nb;
    k.partials = dalloc(ctx, (size_t)nb * 5);
    // per-ring partials of the diagnostics (2 per ring) and of fb_planet_force (4)
    ctx->d_diag = dalloc(ctx, (size_t)nb * 4);
    if (cudaMallocHost((void **)&ctx->h_diag, (size_t)nb * 4 * sizeof(double)) != cudaSuccess) {
      fb_destroy(ctx);
      return FB_ERR_NOMEM;
    }
  }
  if (cudaMalloc((void **)&ctx->d_ctl, sizeof(fb_ctl)) != cudaSuccess ||
      cudaMallocHost((void **)&ctx->h_ctl, sizeof(fb_ctl)) != cudaSuccess) {
    fb_destroy(ctx);
    return FB_ERR_NOMEM;
  }
  cudaMemset(ctx->d_ctl, 0, sizeof(fb_ctl));
  memset(ctx->h_ctl, 0, sizeof(fb_ctl));
  k.ctl = ctx->d_ctl;
  // scalars
  k.pmin = p->pmin;
  k.pmax = p->pmax;
  k.dphi = (p->pmax - p->pmin) / (double)ns;
  k.invdphi = 1.0 / k.dphi;
  k.omega_frame = p->omegaframe;
  k.corot = p->corotating;
  k.gamma = p->adiabaticindex;
  k.alpha = p->alphaviscosity;
  k.nu_const = p->viscosity;
  k.visc_mode = (p->alphaviscosity != 0.0) ? 1 : (p->viscosity != 0.0 ? 2 : 0);
  k.energy = p->energy_equation;
  k.viscous_heating = p->viscous_heating;
  k.beta_cooling = p->beta_cooling;
  k.fast_transport = p->fast_transport;
  k.wall = p->wall_boundary;
  k.thermal_cooling = p->energy_equation && p->thermal_cooling;
  if (p->energy_equation && p->temppresc && !k.thermal_cooling) {
    // FillPrescTime (Theo.c:200-212) or PRESCTIME0 / pow(Rmed, -1.5)
    std::vector<double> pt(nr);
    for (int i = 0; i < nr; i++)
      pt[i] = (p->viscosity > 0.0) ? p->presctime0 * pow(ctx->g.rmed[i], 2.0 + 2.0 * p->flaringindex)
                                   : p->presctime0 / pow(ctx->g.rmed[i], -1.5);
    k.temppresc = 1;
    k.presc = dtable(ctx, pt.data(), nr);
    if (!k.presc) { fb_destroy(ctx); return FB_ERR_NOMEM; }
  }
  if (p->energy_equation && (p->entropy_diffusion || p->radiative_diffusion)) {
    // thermal diffusion (SubStep0): its scratch fields, and for radiative
    // diffusion the opacity of every substep with ComputeOpacities' constants
    k.ent_diff = p->entropy_diffusion;
    k.rad_diff = p->radiative_diffusion;
    k.diffusivity = p->diffusivity;
    double **tf[] = {&k.td_s, &k.td_t, &k.td_k, &k.td_ent, &k.td_rad};
    for (double **f : tf)
      if (!(*f = dalloc(ctx, nf))) { fb_destroy(ctx); return FB_ERR_NOMEM; }
    if (k.rad_diff) {
      const double um = fb_unit_mass(p), ul = fb_unit_length(p);
      k.sigma_sb = 5.6704e-8 * pow(um, -1) * pow(fb_unit_time(p), 3.) * pow(fb_unit_temperature(p), 4.);
      k.op_constant = p->constant_opacity;
      k.op_imposed = p->imposedconstantopacity;
      k.op_factor = p->factoropacities;
      k.op_utemp = fb_unit_temperature(p);
      k.op_umass = um;
      k.op_invl3 = pow(ul, -3.);
      k.op_conv = 0.1 * pow(ul, -2.0) * pow(um, 1.0);
      if (!k.opacity && !(k.opacity = dalloc(ctx, nf))) { fb_destroy(ctx); return FB_ERR_NOMEM; }
    }
    if (k.rad_diff == 2) {
      k.sor_grid = fb_sor_grid();
      if (k.sor_grid < 1) { set_err(ctx, "no resident CTA for the radiative diffusion solver"); fb_destroy(ctx); return FB_ERR_CUDA; }
      for (int q = 0; q < 6; q++)
        if (!(k.sor_c[q] = dalloc(ctx, nf))) { fb_destroy(ctx); return FB_ERR_NOMEM; }
      k.sor_part = dalloc(ctx, (size_t)3 * k.sor_grid);
      k.sor_bar = (unsigned int *)dalloc(ctx, 1);
      if (!k.sor_part || !k.sor_bar) { fb_destroy(ctx); return FB_ERR_NOMEM; }
    }
  }
  if (k.thermal_cooling) {
    // sigma_SB in code units (LowTasks.c:215)
    k.sigma_sb = 5.6704e-8 * pow(fb_unit_mass(p), -1) * pow(fb_unit_time(p), 3.) * pow(fb_unit_temperature(p), 4.);
    if (!k.opacity) k.opacity = dalloc(ctx, nf);
    if (!k.opacity) { fb_destroy(ctx); return FB_ERR_NOMEM; }
    k.irradiation = p->stellar_irradiation;
    if (k.irradiation) {  // per ring, as SubStep3 evaluates them (SourceEuler.c:1204-1268)
      const double um = fb_unit_mass(p), ul = fb_unit_length(p), ut = fb_unit_time(p);
      const double Lstar = p->stellarluminosity * 3.8e26 * pow(um, -1.0) * pow(ul, -2.0) * pow(ut, 3.0);
      std::vector<double> irr(nr);
      for (int i = 0; i < nr; i++)
        irr[i] = (k.irradiation == 1)
                     ? (p->backgroundtemperature / fb_unit_temperature(p)) * pow(ctx->g.rmed[i], p->slopebackgroundtemperature)
                     : Lstar / 4.0 / M_PI / ctx->g.rmed[i] / ctx->g.rmed[i];
      k.irr_ring = dtable(ctx, irr.data(), nr);
      if (!k.irr_ring) { fb_destroy(ctx); return FB_ERR_NOMEM; }
    }
  }
  k.open_inner = p->open_inner;
  k.kn_open = p->kn_open;
  k.non_reflecting = p->non_reflecting;
  k.sigmaslope = p->sigmaslope;
  if (p->mhd_lsa && p->nbturbmodes > 0) {  // turbulent potential (src/turb.c)
    k.lsa = 1;
    k.lsa_nm = p->nbturbmodes;
    k.lsa_highm = p->high_m_cutoff;
    k.lsa_gamma = p->gammaturb;
    k.lsa_speedup = p->lsamodespeedup;
    k.lsa_rmin = p->turbrmin;
    k.lsa_rmax = p->turbrmax;
    k.cav_rmin = p->cavityradius - p->cavitywidth * p->aspectratio;  // turb.c:82-83
    k.cav_rmax = p->cavityradius + p->cavitywidth * p->aspectratio;
    k.cav_ratio = p->cavityratio;
    k.lsa_st = (fb_lsa *)dalloc(ctx, (sizeof(fb_lsa) + sizeof(double) - 1) / sizeof(double));
    k.lsa_cs = dalloc(ctx, (size_t)2 * k.lsa_nm * ns);
    k.lsa_g = dalloc(ctx, (size_t)k.lsa_nm * nr);
    if (!k.lsa_st || !k.lsa_cs || !k.lsa_g) { fb_destroy(ctx); return FB_ERR_NOMEM; }
    const unsigned long long x0 = fb_rand48_state(0, 0);  // every tf = 0: all modes drawn at the first substep
    cudaMemcpy(&k.lsa_st->x, &x0, sizeof x0, cudaMemcpyHostToDevice);
  }
  if (p->non_reflecting) {
    k.edge_buf = dalloc(ctx, (size_t)3 * ns);
    if (!k.edge_buf) { fb_destroy(ctx); return FB_ERR_NOMEM; }
  }
  if (p->open_inner || p->non_reflecting) {  // the edges' constants, as the reference evaluates them
    const fb_geom &gg = ctx->g;
    k.ob_vt1 = sqrt(gg.rmed[2] / gg.rmed[1]);
    k.ob_vt0 = sqrt(gg.rmed[2] / gg.rmed[0]);
    k.ob_vtout = pow(gg.rmed[nr - 1] / gg.rmed[nr - 2], -0.5);
    k.nrb_om1 = pow(gg.rinf[1], -1.5);
    k.nrb_omn2 = pow(gg.rinf[nr - 2], -1.5);
    k.nrb_csinit0 = sqrt(p->adiabaticindex) * p->aspectratio * pow(gg.rmed[0], -0.5 + p->flaringindex);
    k.nrb_csinit1 = sqrt(p->adiabaticindex) * p->aspectratio * pow(gg.rmed[1], -0.5 + p->flaringindex);
    k.radii0 = gg.radii[0];
    k.radiin = gg.radii[nr];
  }
  k.evanescent = p->evanescent;
  k.add_floors = p->add_floors;
  k.damp_axi = p->damp_to_axi;
  k.zero_vrad = p->zero_vrad_bc;
  k.floordens = p->densityfloor;
  k.wkzrmin = p->wkzrmin;
  k.wkzrmax = p->wkzrmax;
  k.indirect_term = p->indirect_term;
  k.discard_gas_it = p->discard_gas_indirect_term;
  k.alt_gas_it = p->alternative_gas_indirect_term;
  k.exclude_hill = p->exclude_hill;
  k.roche = (p->rochesmoothing != 0.0);
  k.forced_circular = p->forced_circular;
  k.indirect_smoothing = p->indirecttermsmoothing;
  k.rochesmoothing = p->rochesmoothing;
  k.thicksmoothing = p->thicknesssmoothing;
  k.aspectratio = p->aspectratio;
  k.flaringindex = p->flaringindex;
  k.masstaper = p->masstaper;
  k.self_gravity = p->self_gravity;
  k.transport_only = 0;
  k.cell_bs = 128;  // launch shapes: automatic until tuned
  k.azi_E = 0;
  k.rad_tx = 0;
  k.rad_chunk = 0;
  ctx->substep_cap = 1000000;
  {
    const char *cap = getenv("FB_MAX_SUBSTEPS");
    if (cap && atoi(cap) > 0) ctx->substep_cap = atoi(cap);
  }
  if (getenv("FB_NO_GRAPH")) ctx->graph_state = -1;
  if (p->nbpart > 0) {
    rc = dust_create(ctx);
    if (rc) { fb_destroy(ctx); return rc; }
  }
  if (p->self_gravity) {
    rc = fb_sg_create(&ctx->sg, p, &ctx->g, ctx->st);
    if (rc) { set_err(ctx, "self-gravity setup failed (%d)", rc); fb_destroy(ctx); return rc; }
  }
  if (cudaDeviceSynchronize() != cudaSuccess) { fb_destroy(ctx); return FB_ERR_CUDA; }
  *out = ctx;
  return FB_OK;
}

extern "C" int fb_destroy(fb_ctx *ctx)
{
  if (!ctx) return FB_OK;
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  if (ctx->h_dc) cudaFreeHost(ctx->h_dc);
  if (ctx->sg) fb_sg_destroy(ctx->sg);
  for (void *p : ctx->allocs) cudaFree(p);
  if (ctx->d_ctl) cudaFree(ctx->d_ctl);
  if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
  if (ctx->h_diag) cudaFreeHost(ctx->h_diag);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_planets) cudaEventDestroy(ctx->ev_planets);
  if (ctx->st_planets) cudaStreamDestroy(ctx->st_planets);
  if (ctx->ev_sg_fork) cudaEventDestroy(ctx->ev_sg_fork);
  if (ctx->ev_sg_done) cudaEventDestroy(ctx->ev_sg_done);
  if (ctx->ev_vm_fork) cudaEventDestroy(ctx->ev_vm_fork);
  if (ctx->ev_vm_done) cudaEventDestroy(ctx->ev_vm_done);
  if (ctx->st_sg) cudaStreamDestroy(ctx->st_sg);
  for (auto &e : ctx->pev) cudaEventDestroy(e);
  if (ctx->gdt_exec) cudaGraphExecDestroy(ctx->gdt_exec);
  if (ctx->gdt) cudaGraphDestroy(ctx->gdt);
  if (ctx->st) cudaStreamDestroy(ctx->st);
  fb_geom_free(&ctx->g);
  delete ctx;
  return FB_OK;
}

// ------------------------------------------------------------ upload
__global__ void k_fill_cs_iso(KP k)
{
  const size_t n = (size_t)k.nr * k.ns;
  for (size_t l = (size_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += (size_t)gridDim.x * blockDim.x)
    k.cs[l] = k.cs_ring[l / k.ns];
}

extern "C" int fb_upload(fb_ctx *ctx, const fb_state *s, const fb_profiles *prof)
{
  if (!ctx || !s) return FB_ERR_INVALID;
  KP &k = ctx->k;
  const size_t bytes = ctx->nf * sizeof(double);
  const int nr = ctx->nr;
  if (s->dens) CK(cudaMemcpyAsync(k.rho, s->dens, bytes, cudaMemcpyHostToDevice, ctx->st));
  if (s->vrad) CK(cudaMemcpyAsync(k.vr, s->vrad, bytes, cudaMemcpyHostToDevice, ctx->st));
  if (s->vtheta) CK(cudaMemcpyAsync(k.vt, s->vtheta, bytes, cudaMemcpyHostToDevice, ctx->st));
  if (s->energy) CK(cudaMemcpyAsync(k.e, s->energy, bytes, cudaMemcpyHostToDevice, ctx->st));
  if (prof) {
    if (prof->sigma_med) {
      CK(cudaMemcpyAsync((void *)k.sigmamed, prof->sigma_med, nr * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
      ctx->h_supp.assign(nr, 0.0);
      for (int i = 0; i < nr; i++)  // SourceEuler.c:933
        ctx->h_supp[i] = ctx->p.imposeddiskdrift * 0.5 * pow(ctx->g.rmed[i], -2.5) * ctx->p.sigma0 / prof->sigma_med[i];
      CK(cudaMemcpyAsync((void *)k.supp_torque, ctx->h_supp.data(), nr * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    }
    if (prof->energy_med) CK(cudaMemcpyAsync((void *)k.energymed, prof->energy_med, nr * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    if (prof->vtheta_med) CK(cudaMemcpyAsync((void *)k.vthetamed, prof->vtheta_med, nr * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    if (prof->vrad_med) CK(cudaMemcpyAsync((void *)k.vradmed, prof->vrad_med, nr * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    if (prof->global_soundspeed) CK(cudaMemcpyAsync(k.gcs, prof->global_soundspeed, nr * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  }
  if (!ctx->p.energy_equation) {
    k_fill_cs_iso<<<256, 256, 0, ctx->st>>>(k);
  } else {
    fb_launch_soundspeed(k, 0, ctx->st);
  }
  if (k.thermal_cooling || k.rad_diff) {
    // the opacity of the uploaded state, which the step keeps, as the
    // reference computes it once in InitEuler (SourceEuler.c:275)
    const fb_params *pp = &ctx->p;
    const double um = fb_unit_mass(pp), ul = fb_unit_length(pp);
    fb_launch_opacity(k, pp->constant_opacity, pp->imposedconstantopacity, pp->factoropacities,
                      fb_unit_temperature(pp), um, pow(ul, -3.), 0.1 * pow(ul, -2.0) * pow(um, 1.0), ctx->st);
  }
  // scalar state
  fb_ctl *c = ctx->h_ctl;
  CK(cudaStreamSynchronize(ctx->st));
  CK(cudaMemcpy(c, ctx->d_ctl, sizeof(fb_ctl), cudaMemcpyDeviceToHost));
  c->physical_time = s->physical_time;
  c->physical_time_initial = s->physical_time_initial;
  c->omega_frame = s->omega_frame;
  c->lost_mass = s->lost_mass;
  if (!ctx->uploaded) {  // the implicit solver's statics (SourceEuler.c:43, 47)
    c->sor_omega = FB_SOR_OMEGA0;
    c->sor_niterbuf = FB_SOR_MAXITS;
  }
  c->mindt = s->mindt;
  c->maxdt = s->maxdt;
  for (int q = 0; q < 3; q++) {
    c->bary_x[q] = s->stardiscbarycenter_x[q];
    c->bary_y[q] = s->stardiscbarycenter_y[q];
  }
  const fb_planets &pl = s->planets;
  if (pl.nb < 0 || pl.nb > FB_MAX_PLANETS) return FB_ERR_INVALID;
  c->np = pl.nb;
  for (int q = 0; q < pl.nb; q++) {
    if (pl.acc[q] > 1e-10) { set_err(ctx, "planet accretion is not supported"); return FB_ERR_UNSUPPORTED; }
    if (pl.feeldisk[q]) { set_err(ctx, "planets feeling the disc are not supported"); return FB_ERR_UNSUPPORTED; }
    if (pl.binary[q]) { set_err(ctx, "binary planets are not supported"); return FB_ERR_UNSUPPORTED; }
    c->pm[q] = pl.mass[q];
    c->px[q] = pl.x[q];
    c->py[q] = pl.y[q];
    c->pvx[q] = pl.vx[q];
    c->pvy[q] = pl.vy[q];
    c->pacc[q] = pl.acc[q];
    c->pinit[q] = pl.initial_mass[q];
    c->pfinal[q] = pl.final_mass[q];
    c->pfeelothers[q] = pl.feelothers[q];
  }
  if (!ctx->p.corotating && ctx->p.omegaframe != s->omega_frame) {
    set_err(ctx, "OmegaFrame must stay OMEGAFRAME (non-rotating frame)");
    return FB_ERR_UNSUPPORTED;
  }
  CK(cudaMemcpy(ctx->d_ctl, c, sizeof(fb_ctl), cudaMemcpyHostToDevice));
  ctx->uploaded = 1;
  return FB_OK;
}

// ------------------------------------------------------------ one DT
// One substep (SourceEuler.c:398-716).  STAGE() records an event before a
// stage when profiling and counts the kernel launches it issues.
#define STAGE(id, nlaunch, call)                                 \
  do {                                                           \
    if (ctx->profiling && npt < FB_PROFILE_POINTS - 1) {         \
      cudaEventRecord(ctx->pev[npt], s);                         \
      ctx->pseq[npt] = (id);                                     \
      npt++;                                                     \
    }                                                            \
    call;                                                        \
    ctx->launches += (nlaunch);                                  \
    ctx->pcount[id] += (nlaunch);                                \
  } while (0)

static int enqueue_substep(fb_ctx *ctx)
{
  KP &k = ctx->k;
  cudaStream_t s = ctx->st;
  int npt = 0;
  // The self-gravity convolution reads only the density, which no kernel
  // changes before the transport: outside the per-stage profile it runs on
  // a branch of its own from the start of the substep, beside the CFL,
  // potential and SubStep1 kernels, and joins before its velocity kicks.
  const bool sg_branch = k.self_gravity && !ctx->profiling;
  if (sg_branch) {
    cudaEventRecord(ctx->ev_sg_fork, s);
    cudaStreamWaitEvent(ctx->st_sg, ctx->ev_sg_fork, 0);
    fb_sg_rows_fwd(ctx->sg, k, k.rho, ctx->st_sg);
    fb_sg_cols(ctx->sg, ctx->st_sg);
    fb_sg_rows_inv(ctx->sg, k, k.rho, ctx->st_sg);
    cudaEventRecord(ctx->ev_sg_done, ctx->st_sg);
    ctx->launches += 3;
    ctx->pcount[ST_SG] += 1;
    ctx->pcount[ST_SGCOLS] += 1;
    ctx->pcount[ST_SGINV] += 1;
  }
  // explicit radiative diffusion: the opacity of the substep's starting
  // state, which ConditionCFL and ComputeRadiativeDiffusion both compute
  // (SourceEuler.c:1326, 1809) and SubStep3's cooling then uses
  if (k.energy && k.rad_diff == 1) {
    STAGE(ST_CFL, 1, fb_launch_opacity_now(k, s));
    STAGE(ST_CFL, 1, fb_launch_td_cfl(k, s));
  }
  STAGE(ST_CFL, 1, fb_launch_cfl(k, s));  // ConditionCFL + the controller (last CTA)
  if (k.corot) {
    // corotating frame: FillForcesArrays' turbulent modes still see the old
    // OmegaFrame; then the planets' step sets the new one and CorrectVtheta
    // applies its change before the gas update (SourceEuler.c:476-525)
    if (k.lsa) STAGE(ST_POT, 2, fb_launch_lsa_modes(k, s));
    STAGE(ST_CFL, 1, fb_launch_planets(k, NULL, s));
    STAGE(ST_CFL, 1, fb_launch_correct_vtheta(k, s));
    cudaEventRecord(ctx->ev_planets, s);
  } else {
    // the planets' step on a branch of its own: no gas kernel of the substep
    // reads the positions it writes; joined before the particles' velocity
    // update, else at the end of the substep
    cudaEventRecord(ctx->ev_fork, s);
    cudaStreamWaitEvent(ctx->st_planets, ctx->ev_fork, 0);
    fb_launch_planets(k, ctx->has_dust ? &ctx->pp : NULL, ctx->st_planets);
    cudaEventRecord(ctx->ev_planets, ctx->st_planets);
    ctx->launches += 1;
    ctx->pcount[ST_CFL] += 1;
  }
  // particles after the planets' RK5 step and before the gas update
  // (SourceEuler.c:504-531)
  if (ctx->has_dust)
    STAGE(ST_DUST, fb_dust_launches(ctx->pp), fb_launch_dust_substep(k, ctx->pp, s, ctx->ev_planets));
  // SubStep0: thermal diffusion, before the sound speed (SourceEuler.c:577-586)
  if (k.energy && (k.ent_diff || k.rad_diff)) {
    int n0 = 0;  // the stage's kernel launches
    STAGE(ST_SUB0, n0, n0 = fb_launch_substep0(k, s));
  }
  if (k.energy) STAGE(ST_SOUND, 1, fb_launch_soundspeed(k, k.visc_mode == 1, s));
  if (k.lsa && !k.corot) STAGE(ST_POT, 2, fb_launch_lsa_modes(k, s));  // the turbulent modes at the substep's start
  STAGE(ST_POT, 1, fb_launch_potential(k, s));
  if (k.lsa) STAGE(ST_POT, 1, fb_launch_lsa_add(k, s));
  STAGE(ST_SUB1, 1, fb_launch_substep1(k, s));
  if (k.self_gravity) {
    if (sg_branch) {
      cudaStreamWaitEvent(s, ctx->ev_sg_done, 0);
    } else {
      STAGE(ST_SG, 1, fb_sg_rows_fwd(ctx->sg, k, k.rho, s));
      STAGE(ST_SGCOLS, 1, fb_sg_cols(ctx->sg, s));
      STAGE(ST_SGINV, 1, fb_sg_rows_inv(ctx->sg, k, k.rho, s));
    }
    STAGE(ST_SGUPD, 1, fb_sg_update_velocities(k, s));
  }
  if (k.visc_mode) {
    STAGE(ST_VTERMS, 1, fb_launch_viscous_terms(k, k.vri, k.vti, s));
    STAGE(ST_VUPDATE, 1, fb_launch_viscous_update(k, k.vri, k.vti, 0.0, s));
  }
  STAGE(ST_SUB2, 1, fb_launch_substep2(k, s));
  // the tile variant's ring means of vtheta, which SubStep2 has just
  // written for the last time before the transport: on a branch beside
  // SubStep3 and the radial pass (in line when profiling stage by stage)
  const bool vm_branch = !ctx->profiling && fb_azi_launches(k) == 2;
  if (vm_branch) {
    cudaEventRecord(ctx->ev_vm_fork, s);
    cudaStreamWaitEvent(ctx->st_sg, ctx->ev_vm_fork, 0);
    fb_launch_azi_vmed(k, 0.0, ctx->st_sg);
    cudaEventRecord(ctx->ev_vm_done, ctx->st_sg);
    ctx->launches += 1;
    ctx->pcount[ST_TVMED] += 1;
  }
  if (k.energy) STAGE(ST_SUB3, 1, fb_launch_substep3(k, s));  // with the stresses of the new velocities
  STAGE(ST_TRAD, 1, fb_launch_transport_radial(k, 0.0, s));
  if (vm_branch) {
    cudaStreamWaitEvent(s, ctx->ev_vm_done, 0);
    STAGE(ST_TAZI, 1, fb_launch_transport_azimuthal(k, 0.0, s, true));
  } else {
    // the tile variant's ring means as a stage of their own, then the pass
    if (fb_azi_launches(k) == 2) STAGE(ST_TVMED, 1, fb_launch_azi_vmed(k, 0.0, s));
    STAGE(ST_TAZI, 1, fb_launch_transport_azimuthal(k, 0.0, s, true));
  }
  STAGE(ST_TVR, 1, fb_launch_transport_vr(k, s));
  if (k.open_inner || k.non_reflecting) {
    // ApplyBoundaryCondition's other edges (SideEuler.c:1102-1131); the
    // non-reflecting edge reads the planets' new positions and, with the
    // energy equation, the sound speed of the transported state
    if (k.non_reflecting && !ctx->has_dust) cudaStreamWaitEvent(s, ctx->ev_planets, 0);
    if (k.non_reflecting && k.energy) STAGE(ST_TVR, 1, fb_launch_soundspeed(k, 0, s));
    STAGE(ST_TVR, 1, fb_launch_edges(k, s));
  }
  if (k.evanescent && k.n_damp_rings > 0) STAGE(ST_DAMP, 1, fb_launch_damping(k, 0.0, s));
  if (!ctx->has_dust) cudaStreamWaitEvent(s, ctx->ev_planets, 0);
  if (ctx->profiling) {
    cudaEventRecord(ctx->pev[npt], s);
    ctx->pseq[npt] = -1;
    npt++;
  }
  return npt;
}

// The start of one DT, before the substep loop; returns the kernel launches.
static int enqueue_dt_prelude(fb_ctx *ctx)
{
  KP &k = ctx->k;
  cudaStream_t s = ctx->st;
  int n = 1;
  fb_launch_begin_dt(k, ctx->p.dt, s);
  if (ctx->has_dust && ctx->sg) {
    // main.c:307-316: before every DT the reference's main loop recomputes
    // the self-gravity field (SoftWriting = No), which sets the RadSGAcc /
    // AziSGAcc grids the first substep's particles read
    fb_sg_accel(ctx->sg, k, k.rho, s);
    fb_sg_update_velocities(k, s, 1);
    n += fb_sg_launches(ctx->sg);
  }
  if (k.energy) {  // SourceEuler.c:344-350
    fb_launch_soundspeed(k, 0, s);
    n += 1;
  }
  if (ctx->has_dust) n += fb_launch_dust_sort(k, ctx->pp, s);  // processing order only
  return n;
}

// Captures one DT as a graph: WHILE(cond) { substep; cond = !done }.  The
// kernels read dt and the planets from the device control block, so one
// capture serves every substep and every DT.
static int build_dt_graph_once(fb_ctx *ctx);
// Without programmatic dependent launch when a driver refuses it in a graph.
static int build_dt_graph(fb_ctx *ctx)
{
  int rc = build_dt_graph_once(ctx);
  if (rc == FB_ERR_CUDA && fb_pdl) {
    fb_pdl = 0;
    rc = build_dt_graph_once(ctx);
  }
  return rc;
}

static int build_dt_graph_once(fb_ctx *ctx)
{
  cudaGraph_t g = NULL, body = NULL;
  cudaGraphConditionalHandle h;
  cudaGraphNode_t node;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return FB_ERR_CUDA;
  if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
    cudaGraphDestroy(g);
    return FB_ERR_CUDA;
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if (cudaGraphAddNode(&node, g, NULL, 0, &cp) != cudaSuccess) {
    cudaGraphDestroy(g);
    return FB_ERR_CUDA;
  }
  body = cp.conditional.phGraph_out[0];
  const long long l0 = ctx->launches;
  const int prof = ctx->profiling;
  ctx->profiling = 0;
  cudaError_t e = cudaStreamBeginCaptureToGraph(ctx->st, body, NULL, NULL, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    enqueue_substep(ctx);
    fb_launch_loop_cond(ctx->k, h, ctx->substep_cap, ctx->st);
    e = cudaStreamEndCapture(ctx->st, &body);
  }
  ctx->profiling = prof;
  ctx->launches_per_substep = ctx->launches - l0 + 1;
  ctx->launches = l0;
  for (int q = 0; q < FB_NSTAGE; q++) ctx->pcount[q] = 0;
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return FB_ERR_CUDA;
  }
  if (cudaGraphInstantiate(&ctx->gdt_exec, g, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return FB_ERR_CUDA;
  }
  ctx->gdt = g;
  return FB_OK;
}

static void profile_collect(fb_ctx *ctx, int npt)
{
  for (int q = 0; q + 1 < npt; q++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->pev[q], ctx->pev[q + 1]) == cudaSuccess && ctx->pseq[q] >= 0)
      ctx->pms[ctx->pseq[q]] += ms;
  }
}

extern "C" long long fb_kernel_launches(const fb_ctx *ctx) { return ctx ? ctx->launches : -1; }

extern "C" int fb_profile(fb_ctx *ctx, int enable)
{
  if (!ctx) return FB_ERR_INVALID;
  if (enable && ctx->pev.empty()) {
    ctx->pev.resize(FB_PROFILE_POINTS);  // the recorded points of one substep, with room to spare
    ctx->pseq.resize(FB_PROFILE_POINTS);
    for (auto &e : ctx->pev) CK(cudaEventCreate(&e));
  }
  ctx->profiling = enable ? 1 : 0;
  for (int q = 0; q < FB_NSTAGE; q++) { ctx->pms[q] = 0.0; ctx->pcount[q] = 0; }
  return FB_OK;
}

extern "C" int fb_profile_read(const fb_ctx *ctx, int idx, const char **name, double *ms, long long *launches)
{
  if (!ctx) return FB_ERR_INVALID;
  if (idx < 0 || idx >= FB_NSTAGE) return FB_NSTAGE;
  if (name) *name = stage_names[idx];
  if (ms) *ms = ctx->pms[idx];
  if (launches) *launches = ctx->pcount[idx];
  return FB_NSTAGE;
}

// The DetectCrash bookkeeping of one DT (SourceEuler.c:545-566), and the
// disc's pull on the star that AlgoGas leaves in DiskOnPrimaryAcceleration.
static void report_crash(const fb_ctl *c, fb_step_report *rep)
{
  rep->disk_on_primary[0] = c->disk_acc_x;  // DiskOnPrimaryAcceleration of the last substep
  rep->disk_on_primary[1] = c->disk_acc_y;
  rep->disk_on_primary_alt[0] = c->disk_acc_alt_x;
  rep->disk_on_primary_alt[1] = c->disk_acc_alt_y;
  rep->crashes = c->crashes;
  rep->crash_substeps = c->crash_substeps;
  rep->neg_density_substeps = c->neg_dens_substeps;
  rep->crash_time = c->crashes > 0 ? c->crash_time : 0.0;
}

extern "C" int fb_algogas(fb_ctx *ctx, fb_step_report *rep)
{
  if (!ctx) return FB_ERR_INVALID;
  if (!ctx->uploaded) return FB_ERR_STATE;
  if (ctx->has_dust && !ctx->dust_uploaded) {
    set_err(ctx, "NBPART > 0: upload the particles (fb_dust_upload) before the first DT");
    return FB_ERR_STATE;
  }
  cudaStream_t s = ctx->st;
  CK(cudaEventRecord(ctx->ev0, s));
  ctx->launches += enqueue_dt_prelude(ctx);
  int status = FB_OK;
  const int cap = ctx->substep_cap;
  if (!ctx->profiling && ctx->graph_state == 0) ctx->graph_state = (build_dt_graph(ctx) == FB_OK) ? 1 : -1;
  if (!ctx->profiling && ctx->graph_state == 1) {
    CK(cudaGraphLaunch(ctx->gdt_exec, s));
    CK(cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, sizeof(fb_ctl), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    status = ctx->h_ctl->status;
    ctx->launches += ctx->launches_per_substep * (long long)ctx->h_ctl->substeps;
  } else for (int it = 0; it < cap; it++) {
    int npt = enqueue_substep(ctx);
    CK(cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, sizeof(fb_ctl), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (ctx->profiling) profile_collect(ctx, npt);
    if (ctx->h_ctl->status) { status = ctx->h_ctl->status; break; }
    if (ctx->h_ctl->done) break;
    if (it == cap - 1) status = FB_ERR_SUBSTEPS;
  }
  CK(cudaEventRecord(ctx->ev1, s));
  CK(cudaEventSynchronize(ctx->ev1));
  CK(cudaGetLastError());
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  const fb_ctl *c = ctx->h_ctl;
  if (rep) {
    rep->substeps = c->substeps;
    rep->status = status;
    rep->physical_time = c->physical_time;
    rep->mindt = c->mindt;
    rep->maxdt = c->maxdt;
    rep->lost_mass = c->lost_mass;
    rep->gpu_ms = ms;
    report_crash(c, rep);
  }
  if (status) {
    set_err(ctx, "AlgoGas stopped: %s", fb_strerror(status));
  } else if (c->crash_substeps > 0) {
    // the DT ran to its end, as the reference's does after a crash
    set_err(ctx, "DetectCrash: negative energy in %d substep(s) of this DT; first crash at time %.12g",
            c->crash_substeps, c->crash_time);
    status = FB_ERR_NEGATIVE;
    if (rep) rep->status = status;
  }
  return status;
}

// ------------------------------------------------------------ download
extern "C" int fb_download(fb_ctx *ctx, fb_state *s, unsigned mask)
{
  if (!ctx || !s) return FB_ERR_INVALID;
  KP &k = ctx->k;
  const size_t bytes = ctx->nf * sizeof(double);
  if ((mask & FB_F_DENS) && s->dens) CK(cudaMemcpyAsync(s->dens, k.rho, bytes, cudaMemcpyDeviceToHost, ctx->st));
  if ((mask & FB_F_VRAD) && s->vrad) CK(cudaMemcpyAsync(s->vrad, k.vr, bytes, cudaMemcpyDeviceToHost, ctx->st));
  if ((mask & FB_F_VTHETA) && s->vtheta) CK(cudaMemcpyAsync(s->vtheta, k.vt, bytes, cudaMemcpyDeviceToHost, ctx->st));
  if ((mask & FB_F_ENERGY) && s->energy) CK(cudaMemcpyAsync(s->energy, k.e, bytes, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, sizeof(fb_ctl), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  const fb_ctl *c = ctx->h_ctl;
  s->physical_time = c->physical_time;
  s->physical_time_initial = c->physical_time_initial;
  s->omega_frame = c->omega_frame;
  s->lost_mass = c->lost_mass;
  s->mindt = c->mindt;
  s->maxdt = c->maxdt;
  for (int q = 0; q < 3; q++) {
    s->stardiscbarycenter_x[q] = c->bary_x[q];
    s->stardiscbarycenter_y[q] = c->bary_y[q];
  }
  s->planets.nb = c->np;
  for (int q = 0; q < c->np; q++) {
    s->planets.mass[q] = c->pm[q];
    s->planets.x[q] = c->px[q];
    s->planets.y[q] = c->py[q];
    s->planets.vx[q] = c->pvx[q];
    s->planets.vy[q] = c->pvy[q];
  }
  return FB_OK;
}

extern "C" int fb_download_crash(fb_ctx *ctx, fb_state *s, double *crash_time)
{
  if (!ctx || !s) return FB_ERR_INVALID;
  const fb_ctl *c = ctx->h_ctl;
  if (!ctx->k.crash_snap || !c->crash_snapped) {
    set_err(ctx, "no crash has been detected");
    return FB_ERR_STATE;
  }
  const size_t n = (size_t)ctx->nr * ctx->ns;
  double *dst[4] = {s->dens, s->vrad, s->vtheta, s->energy};
  for (int q = 0; q < 4; q++)
    if (dst[q]) CK(cudaMemcpyAsync(dst[q], ctx->k.crash_snap + q * n, n * sizeof(double), cudaMemcpyDeviceToHost,
                                   ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (crash_time) *crash_time = c->crash_time;
  return FB_OK;
}

extern "C" int fb_download_derived(fb_ctx *ctx, int which, double *out)
{
  if (!ctx || !out || which < 0 || which > 7) return FB_ERR_INVALID;
  double *tmp = NULL;
  CK(cudaMallocAsync((void **)&tmp, ctx->nf * sizeof(double), ctx->st));
  CK(cudaMemsetAsync(tmp, 0, ctx->nf * sizeof(double), ctx->st));
  fb_launch_derived(ctx->k, which, tmp, ctx->st);
  CK(cudaMemcpyAsync(out, tmp, ctx->nf * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaFreeAsync(tmp, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return FB_OK;
}

extern "C" int fb_lsa_stream(fb_ctx *ctx, unsigned long long *x, int set)
{
  if (!ctx || !x) return FB_ERR_INVALID;
  if (!ctx->k.lsa) {
    set_err(ctx, "fb_lsa_stream: the context has no turbulent potential (MHD L)");
    return FB_ERR_STATE;
  }
  unsigned long long *dx = &ctx->k.lsa_st->x;
  if (set) {
    const unsigned long long v = *x & 0xFFFFFFFFFFFFull;
    CK(cudaMemcpyAsync(dx, &v, sizeof v, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  } else {
    CK(cudaMemcpyAsync(x, dx, sizeof *x, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  return FB_OK;
}

extern "C" int fb_diagnostics(fb_ctx *ctx, double *mass, double *momentum)
{
  if (!ctx) return FB_ERR_INVALID;
  const int nb = ctx->k.n_partial_blocks;
  fb_launch_diag(ctx->k, ctx->d_diag, ctx->st);
  CK(cudaMemcpyAsync(ctx->h_diag, ctx->d_diag, (size_t)nb * 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  double m = 0.0, p = 0.0;
  for (int b = 0; b < nb; b++) {
    m += ctx->h_diag[2 * b];
    p += ctx->h_diag[2 * b + 1];
  }
  if (mass) *mass = m;
  if (momentum) *momentum = p;
  return FB_OK;
}

extern "C" int fb_download_sgacc(fb_ctx *ctx, int ring0, int nrings, double *accr, double *acct)
{
  if (!ctx || ring0 < 0 || nrings < 0 || ring0 + nrings > ctx->nr) return FB_ERR_INVALID;
  if (!ctx->sg) return FB_ERR_STATE;
  const size_t off = (size_t)ring0 * ctx->ns, n = (size_t)nrings * ctx->ns * sizeof(double);
  if (accr) CK(cudaMemcpyAsync(accr + off, ctx->k.sg_accr + off, n, cudaMemcpyDeviceToHost, ctx->st));
  if (acct) CK(cudaMemcpyAsync(acct + off, ctx->k.sg_acct + off, n, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return FB_OK;
}

extern "C" int fb_planet_force(fb_ctx *ctx, double x, double y, double rsmoothing, double mass, double *out)
{
  if (!ctx || !out) return FB_ERR_INVALID;
  if (!ctx->uploaded) return FB_ERR_STATE;
  const int nr = ctx->nr;
  // ComputeForce (Force.c:118-119): star-planet distance and Hill radius
  const double a = sqrt(x * x + y * y);
  const double rh = pow(mass / 3., 1. / 3.) * a + 1e-15;
  const double cutoff = ctx->p.excludehillfactor * rh;  // hillcutfactor of k = 1 (dimfxy = 2)
  fb_launch_body_force(ctx->k, x, y, rsmoothing, cutoff, ctx->d_diag, ctx->st);
  ctx->launches += 1;
  CK(cudaMemcpyAsync(ctx->h_diag, ctx->d_diag, (size_t)nr * 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  // the rings in order, each into the inner or the outer sums (Force.c:218-226)
  double fxi[2] = {0., 0.}, fxo[2] = {0., 0.}, fyi[2] = {0., 0.}, fyo[2] = {0., 0.};
  for (int i = 0; i < nr; i++) {
    const double *p = ctx->h_diag + (size_t)i * 4;
    if (ctx->g.rmed[i] < a) {
      fxi[0] += p[0]; fxi[1] += p[1]; fyi[0] += p[2]; fyi[1] += p[3];
    } else {
      fxo[0] += p[0]; fxo[1] += p[1]; fyo[0] += p[2]; fyo[1] += p[3];
    }
  }
  out[0] = fxi[0]; out[1] = fxi[1]; out[2] = fxo[0]; out[3] = fxo[1];
  out[4] = fyi[0]; out[5] = fyi[1]; out[6] = fyo[0]; out[7] = fyo[1];
  return FB_OK;
}

// ------------------------------------------------------------ stages
extern "C" int fb_stage(fb_ctx *ctx, int stage, double dt)
{
  if (!ctx) return FB_ERR_INVALID;
  if (!ctx->uploaded) return FB_ERR_STATE;
  KP k = ctx->k;
  cudaStream_t s = ctx->st;
  switch (stage) {
    case FB_STAGE_TRANSPORT:
      if (!(dt > 0.0)) return FB_ERR_INVALID;
      k.transport_only = 1;
      fb_launch_transport(k, dt, s);
      break;
    case FB_STAGE_VISCOSITY:
      if (!(dt > 0.0)) return FB_ERR_INVALID;
      if (k.energy) fb_launch_soundspeed(k, k.visc_mode == 1, s);
      fb_launch_viscous_terms(k, k.vr, k.vt, s);
      fb_launch_viscous_update(k, k.vr, k.vt, dt, s);
      break;
    case FB_STAGE_BOUNDARY:
      fb_launch_boundary_only(k, s);
      if (k.open_inner || k.non_reflecting) {  // ApplyBoundaryCondition's other edges, as in the substep
        if (k.non_reflecting && k.energy) fb_launch_soundspeed(k, 0, s);
        fb_launch_edges(k, s);
      }
      break;
    case FB_STAGE_DAMPING:
      if (!(dt > 0.0)) return FB_ERR_INVALID;
      fb_launch_damping(k, dt, s);
      break;
    case FB_STAGE_SELFGRAV:
      if (!ctx->sg) return FB_ERR_STATE;
      fb_sg_accel(ctx->sg, k, k.rho, s);
      break;
    default:
      return FB_ERR_INVALID;
  }
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return FB_OK;
}

// Initial-state helper for self-gravity: SG acceleration of a host density
// and its azimuthal means (mpi_make1Dprofile of SG_Accr, sgsysinit.c:13-14).
extern "C" int fb_sg_axisym_accel(fb_ctx *ctx, const double *dens, double *axi_out)
{
  if (!ctx || !dens || !axi_out) return FB_ERR_INVALID;
  if (!ctx->sg) return FB_ERR_STATE;
  KP &k = ctx->k;
  const int nr = ctx->nr, ns = ctx->ns;
  CK(cudaMemcpyAsync(k.rho, dens, ctx->nf * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  fb_sg_accel(ctx->sg, k, k.rho, ctx->st);
  std::vector<double> acc((size_t)nr * ns);
  CK(cudaMemcpyAsync(acc.data(), k.sg_accr, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  for (int i = 0; i < nr; i++) {
    double a = 0.0;
    for (int j = 0; j < ns; j++) a += acc[(size_t)i * ns + j];
    a /= (double)ns;
    axi_out[i] = a;
  }
  return FB_OK;
}

// Same as fb_sg_axisym_accel for the density already on the device.
extern "C" int fb_sg_axisym_accel_device(fb_ctx *ctx, double *axi_out)
{
  if (!ctx || !axi_out) return FB_ERR_INVALID;
  if (!ctx->sg) return FB_ERR_STATE;
  if (!ctx->uploaded) return FB_ERR_STATE;
  KP &k = ctx->k;
  const int nr = ctx->nr, ns = ctx->ns;
  fb_sg_accel(ctx->sg, k, k.rho, ctx->st);
  std::vector<double> acc((size_t)nr * ns);
  CK(cudaMemcpyAsync(acc.data(), k.sg_accr, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  for (int i = 0; i < nr; i++) {
    double a = 0.0;
    for (int j = 0; j < ns; j++) a += acc[(size_t)i * ns + j];
    a /= (double)ns;
    axi_out[i] = a;
  }
  return FB_OK;
}

// ------------------------------------------------------------ particles
extern "C" int fb_dust_upload(fb_ctx *ctx, const fb_dust_state *st)
{
  if (!ctx || !st) return FB_ERR_INVALID;
  if (!ctx->has_dust) { set_err(ctx, "context created with NBPART = 0"); return FB_ERR_STATE; }
  if (!ctx->uploaded) { set_err(ctx, "upload the gas state (fb_upload) first"); return FB_ERR_STATE; }
  PP &pp = ctx->pp;
  if (st->n != pp.n || !st->r || !st->th || !st->vr || !st->vth || !st->l || !st->size || !st->stokes)
    return FB_ERR_INVALID;
  if (st->kicks < 0 || st->rng_x > 0xFFFFFFFFFFFFull) return FB_ERR_INVALID;
  if (st->particles_mass != 0.0) {
    set_err(ctx, "a non-zero particle mass needs the dust feedback / dust-fluid paths, not in this build");
    return FB_ERR_UNSUPPORTED;
  }
  const size_t b = (size_t)pp.n * sizeof(double);
  const double *src[] = {st->r, st->th, st->vr, st->vth, st->l, st->size, st->stokes};
  double *dst[] = {pp.r, pp.th, pp.vr, pp.vth, pp.l, pp.size, pp.st};
  for (int f = 0; f < 7; f++) CK(cudaMemcpyAsync(dst[f], src[f], b, cudaMemcpyHostToDevice, ctx->st));
  fb_launch_dust_iota(pp, ctx->st);  // slots in the reference's order until the first sort
  ctx->launches += 1;
  fb_dust_ctl *h = ctx->h_dc;
  memset(h, 0, sizeof *h);
  h->x = st->rng_x;
  h->kicks = st->kicks;
  h->carry_rad = st->carry[0];
  h->carry_phi = st->carry[1];
  h->min_ts = 1e6;
  CK(cudaMemcpyAsync(pp.dc, h, sizeof *h, cudaMemcpyHostToDevice, ctx->st));
  // the interpolation call of main.c:287: Stokes numbers at the uploaded state
  ctx->launches += fb_launch_dust_sort(ctx->k, pp, ctx->st);
  fb_launch_dust_interpolation_only(ctx->k, pp, ctx->st);
  ctx->launches += 1;
  CK(cudaStreamSynchronize(ctx->st));
  CK(cudaGetLastError());
  ctx->dust_uploaded = 1;
  return FB_OK;
}

extern "C" int fb_dust_download(fb_ctx *ctx, fb_dust_state *st)
{
  if (!ctx || !st) return FB_ERR_INVALID;
  if (!ctx->has_dust) return FB_ERR_STATE;
  PP &pp = ctx->pp;
  if (st->n != pp.n) return FB_ERR_INVALID;
  const size_t b = (size_t)pp.n * sizeof(double);
  double *dst[] = {st->r, st->th, st->vr, st->vth, st->l, st->size, st->stokes};
  const double *src[] = {pp.r, pp.th, pp.vr, pp.vth, pp.l, pp.size, pp.st};
  // back in the reference's order through the scratch arrays
  for (int f = 0; f < 7; f++) {
    if (!dst[f]) continue;
    double *tmp = pp.pscratch + (size_t)f * pp.n;
    fb_launch_dust_to_reference_order(pp, src[f], tmp, ctx->st);
    ctx->launches += 1;
    CK(cudaMemcpyAsync(dst[f], tmp, b, cudaMemcpyDeviceToHost, ctx->st));
  }
  CK(cudaMemcpyAsync(ctx->h_dc, pp.dc, sizeof(fb_dust_ctl), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  const fb_dust_ctl *h = ctx->h_dc;
  if (h->err) {
    set_err(ctx, "particle random stream: too few candidate pairs");
    return FB_ERR_INVALID;
  }
  st->rng_x = h->x;
  st->kicks = h->kicks;
  st->carry[0] = h->carry_rad;
  st->carry[1] = h->carry_phi;
  st->particles_mass = 0.0;
  return FB_OK;
}

// ------------------------------------------------------------ diagnostics
extern "C" int fb_vortensity(fb_ctx *ctx, double *field, double *sigma_mean, double *vort_mean)
{
  if (!ctx) return FB_ERR_INVALID;
  if (!ctx->uploaded) return FB_ERR_STATE;
  const int nr = ctx->nr, ns = ctx->ns;
  double *xi = NULL, *means = NULL;
  CK(cudaMallocAsync((void **)&xi, ctx->nf * sizeof(double), ctx->st));
  CK(cudaMallocAsync((void **)&means, 2 * (size_t)nr * sizeof(double), ctx->st));
  CK(cudaMemsetAsync(xi, 0, ctx->nf * sizeof(double), ctx->st));
  fb_launch_vortensity(ctx->k, xi, ctx->st);
  fb_launch_ring_mean(ctx->k.rho, nr, ns, means, ctx->st);
  fb_launch_ring_mean(xi, nr, ns, means + nr, ctx->st);
  ctx->launches += 3;
  if (field) CK(cudaMemcpyAsync(field, xi, ctx->nf * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  if (sigma_mean) CK(cudaMemcpyAsync(sigma_mean, means, nr * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  if (vort_mean) CK(cudaMemcpyAsync(vort_mean, means + nr, nr * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaFreeAsync(xi, ctx->st));
  CK(cudaFreeAsync(means, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return FB_OK;
}

// ------------------------------------------------------------ batches
// Many discs (contexts of any grid size and parameters on one device)
// advanced one DT each by a single graph launch: per disc, the DT prelude
// followed by a conditional WHILE node around its substep, all discs as
// independent branches of one graph so that their kernels overlap on the
// GPU.  No counterpart in the reference, which runs one disc per process.
struct fb_batch {
  std::vector<fb_ctx *> ctxs;
  std::vector<int> prelude;  // kernel launches of each disc's DT prelude
  std::vector<long long> per_substep;
  cudaStream_t st;
  cudaEvent_t ev0, ev1;
  cudaStream_t st_planets;            // branch of the planets' step (k_planets)
  cudaEvent_t ev_fork, ev_planets;    // its start and end within a substep
  cudaStream_t st_sg;                 // branch of the self-gravity convolution
  cudaEvent_t ev_sg_fork, ev_sg_done;
  cudaGraph_t g;
  cudaGraphExec_t ge;
};

extern "C" int fb_batch_destroy(fb_batch *b)
{
  if (!b) return FB_OK;
  if (b->st) cudaStreamSynchronize(b->st);
  if (b->ge) cudaGraphExecDestroy(b->ge);
  if (b->g) cudaGraphDestroy(b->g);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return FB_OK;
}

// One disc of the batch graph: its DT prelude as a child graph, then the
// conditional WHILE node around its substep (captured into the node's body).
static int batch_add_disc(fb_batch *b, fb_ctx *ctx)
{
  cudaStream_t s = ctx->st;
  const long long l0 = ctx->launches;
  const int prof = ctx->profiling;
  ctx->profiling = 0;
  int rc = FB_ERR_CUDA;
  cudaGraph_t pre = NULL;
  cudaGraphNode_t pre_node, loop_node;
  cudaGraphConditionalHandle h;
  cudaGraphNodeParams cp = {};
  int npre = 0;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) goto out;
  npre = enqueue_dt_prelude(ctx);
  if (cudaStreamEndCapture(s, &pre) != cudaSuccess || !pre) goto out;
  if (cudaGraphAddChildGraphNode(&pre_node, b->g, NULL, 0, pre) != cudaSuccess) goto out;
  if (cudaGraphConditionalHandleCreate(&h, b->g, 1, cudaGraphCondAssignDefault) != cudaSuccess) goto out;
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if (cudaGraphAddNode(&loop_node, b->g, &pre_node, 1, &cp) != cudaSuccess) goto out;
  {
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const long long l1 = ctx->launches;
    if (cudaStreamBeginCaptureToGraph(s, body, NULL, NULL, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      goto out;
    enqueue_substep(ctx);
    fb_launch_loop_cond(ctx->k, h, ctx->substep_cap, s);
    if (cudaStreamEndCapture(s, &body) != cudaSuccess) goto out;
    b->prelude.push_back(npre);
    b->per_substep.push_back(ctx->launches - l1 + 1);
  }
  rc = FB_OK;
out:
  if (rc) cudaGetLastError();
  if (pre) cudaGraphDestroy(pre);
  ctx->launches = l0;
  for (int q = 0; q < FB_NSTAGE; q++) ctx->pcount[q] = 0;
  ctx->profiling = prof;
  return rc;
}

extern "C" int fb_batch_create(fb_ctx *const *ctxs, int n, fb_batch **out)
{
  if (!ctxs || n <= 0 || !out) return FB_ERR_INVALID;
  *out = NULL;
  for (int d = 0; d < n; d++) {
    if (!ctxs[d]) return FB_ERR_INVALID;
    if (!ctxs[d]->uploaded || (ctxs[d]->has_dust && !ctxs[d]->dust_uploaded)) return FB_ERR_STATE;
    for (int e = 0; e < d; e++)
      if (ctxs[e] == ctxs[d]) return FB_ERR_INVALID;  // a disc may appear once
  }
  fb_batch *b = new fb_batch();
  b->ctxs.assign(ctxs, ctxs + n);
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
      cudaGraphCreate(&b->g, 0) != cudaSuccess) {
    fb_batch_destroy(b);
    return FB_ERR_CUDA;
  }
  for (int d = 0; d < n; d++) {
    int rc = batch_add_disc(b, ctxs[d]);
    if (rc) { fb_batch_destroy(b); return rc; }
  }
  if (cudaGraphInstantiate(&b->ge, b->g, 0) != cudaSuccess) {
    cudaGetLastError();
    fb_batch_destroy(b);
    return FB_ERR_CUDA;
  }
  *out = b;
  return FB_OK;
}

extern "C" int fb_batch_algogas(fb_batch *b, fb_step_report *reps)
{
  if (!b) return FB_ERR_INVALID;
  const int n = (int)b->ctxs.size();
  fb_ctx *ctx = b->ctxs[0];  // for CK error messages
  // the discs' own streams may still hold work (uploads, single DTs)
  for (fb_ctx *c : b->ctxs) CK(cudaStreamSynchronize(c->st));
  CK(cudaEventRecord(b->ev0, b->st));
  CK(cudaGraphLaunch(b->ge, b->st));
  CK(cudaEventRecord(b->ev1, b->st));
  for (fb_ctx *c : b->ctxs) CK(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(fb_ctl), cudaMemcpyDeviceToHost, b->st));
  CK(cudaStreamSynchronize(b->st));
  CK(cudaGetLastError());
  float ms = 0.f;
  cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  int status = FB_OK;
  for (int d = 0; d < n; d++) {
    fb_ctx *c = b->ctxs[d];
    const fb_ctl *h = c->h_ctl;
    c->launches += b->prelude[d] + b->per_substep[d] * (long long)h->substeps;
    if (h->status && !status) status = h->status;
    if (h->status) set_err(c, "AlgoGas stopped: %s", fb_strerror(h->status));
    if (reps) {
      reps[d].substeps = h->substeps;
      reps[d].status = h->status;
      reps[d].physical_time = h->physical_time;
      reps[d].mindt = h->mindt;
      reps[d].maxdt = h->maxdt;
      reps[d].lost_mass = h->lost_mass;
      reps[d].gpu_ms = ms;  // the whole batch
      report_crash(h, &reps[d]);
    }
    if (!h->status && h->crash_substeps > 0) {  // the disc's DT ran to its end (see fb_algogas)
      set_err(c, "DetectCrash: negative energy in %d substep(s) of this DT; first crash at time %.12g",
              h->crash_substeps, h->crash_time);
      if (reps) reps[d].status = FB_ERR_NEGATIVE;
      if (!status) status = FB_ERR_NEGATIVE;
    }
  }
  return status;
}

// ------------------------------------------------------------ tuning
// Launch shapes of the per-cell, azimuthal and radial kernels.  No
// counterpart in the reference.  fb_tune times candidates on this context's
// own disc (a few substeps each, per-stage CUDA events) from a saved state,
// which it restores afterwards, so tuning does not advance the disc.
static void invalidate_graph(fb_ctx *ctx)
{
  if (ctx->gdt_exec) cudaGraphExecDestroy(ctx->gdt_exec);
  if (ctx->gdt) cudaGraphDestroy(ctx->gdt);
  ctx->gdt_exec = NULL;
  ctx->gdt = NULL;
  if (ctx->graph_state == 1) ctx->graph_state = 0;
}

extern "C" int fb_get_tuning(const fb_ctx *ctx, fb_tuning *t)
{
  if (!ctx || !t) return FB_ERR_INVALID;
  const KP &k = ctx->k;
  t->cell_block = k.cell_bs;
  t->azi_cells_per_thread = k.azi_E > 0 ? k.azi_E : fb_azi_E_auto(k.ns);
  t->rad_columns = k.rad_tx > 0 ? k.rad_tx : 64;
  t->rad_rings = k.rad_chunk > 0 ? k.rad_chunk : fb_rad_chunk_auto(k);
  t->azi_variant = fb_azi_variant(k.ns, k.energy, t->azi_cells_per_thread, k.azi_variant);
  return FB_OK;
}

extern "C" int fb_set_tuning(fb_ctx *ctx, const fb_tuning *t)
{
  if (!ctx || !t) return FB_ERR_INVALID;
  KP &k = ctx->k;
  const int cb = t->cell_block ? t->cell_block : 128;
  if (cb < 32 || cb > 256 || cb % 32) return FB_ERR_INVALID;
  if (t->azi_cells_per_thread && !fb_azi_E_valid(k.ns, k.energy, t->azi_cells_per_thread)) return FB_ERR_INVALID;
  if (t->rad_columns && (t->rad_columns < 32 || t->rad_columns > 128 || t->rad_columns % 32)) return FB_ERR_INVALID;
  if (t->rad_rings < 0 || t->rad_rings > k.nr) return FB_ERR_INVALID;
  const int E = t->azi_cells_per_thread ? t->azi_cells_per_thread : fb_azi_E_auto(k.ns);
  if (t->azi_variant < 0 || t->azi_variant > 8 || !fb_azi_variant(k.ns, k.energy, E, t->azi_variant))
    return FB_ERR_INVALID;
  k.cell_bs = cb;
  k.azi_variant = t->azi_variant;
  k.azi_E = t->azi_cells_per_thread;
  k.rad_tx = t->rad_columns;
  k.rad_chunk = t->rad_rings;
  invalidate_graph(ctx);
  return FB_OK;
}

namespace {
struct Snapshot {
  std::vector<std::pair<void *, size_t>> regions;
  std::vector<void *> copies;
};
}  // namespace

static int snapshot_take(fb_ctx *ctx, Snapshot &sn)
{
  KP &k = ctx->k;
  const size_t nf = ctx->nf * sizeof(double), nr = (size_t)ctx->nr * sizeof(double);
  sn.regions = {{k.rho, nf}, {k.vr, nf}, {k.vt, nf}, {k.e, nf}, {k.cs, nf}, {k.gcs, nr},
                {k.lost0, (size_t)ctx->ns * sizeof(double)}, {ctx->d_ctl, sizeof(fb_ctl)}};
  if (ctx->has_dust) {
    PP &pp = ctx->pp;
    const size_t np = (size_t)pp.n * sizeof(double);
    double *g[] = {k.indpot, k.rgp, k.agp, k.rind, k.aind, k.rsga, k.asga};
    for (double *f : g) sn.regions.push_back({f, nf});
    double *a[] = {pp.r, pp.th, pp.vr, pp.vth, pp.l, pp.size, pp.st};  // permuted by the DT's sort
    for (double *f : a) sn.regions.push_back({f, np});
    sn.regions.push_back({pp.orig, (size_t)pp.n * sizeof(int)});
    sn.regions.push_back({pp.dc, sizeof(fb_dust_ctl)});
  }
  for (auto &r : sn.regions) {
    void *c = NULL;
    if (cudaMalloc(&c, r.second) != cudaSuccess) return FB_ERR_NOMEM;
    sn.copies.push_back(c);
    CK(cudaMemcpyAsync(c, r.first, r.second, cudaMemcpyDeviceToDevice, ctx->st));
  }
  return FB_OK;
}

static int snapshot_restore(fb_ctx *ctx, const Snapshot &sn)
{
  for (size_t q = 0; q < sn.copies.size(); q++)
    CK(cudaMemcpyAsync(sn.regions[q].first, sn.copies[q], sn.regions[q].second, cudaMemcpyDeviceToDevice, ctx->st));
  return FB_OK;
}

static void snapshot_free(Snapshot &sn)
{
  for (void *c : sn.copies) cudaFree(c);
  sn.copies.clear();
}

// Runs `substeps` substeps from the snapshot with per-stage events; returns
// the summed device ms of the stages in `stages` (per substep), or < 0.
static double tune_measure(fb_ctx *ctx, const Snapshot &sn, int substeps, const int *stages, int nst)
{
  if (snapshot_restore(ctx, sn)) return -1.0;
  for (int q = 0; q < FB_NSTAGE; q++) { ctx->pms[q] = 0.0; ctx->pcount[q] = 0; }
  cudaStream_t s = ctx->st;
  const long long l0 = ctx->launches;
  enqueue_dt_prelude(ctx);
  for (int it = 0; it < substeps + 1; it++) {
    if (it == 1)  // the first substep warms caches and is not counted
      for (int q = 0; q < FB_NSTAGE; q++) { ctx->pms[q] = 0.0; ctx->pcount[q] = 0; }
    const int npt = enqueue_substep(ctx);
    if (cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, sizeof(fb_ctl), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      cudaGetLastError();
      return -1.0;
    }
    profile_collect(ctx, npt);
    if (ctx->h_ctl->status) return -1.0;
    if (ctx->h_ctl->done) enqueue_dt_prelude(ctx);  // start another DT from here
  }
  ctx->launches = l0;
  double ms = 0.0;
  for (int q = 0; q < nst; q++) ms += ctx->pms[stages[q]];
  return ms / substeps;
}

extern "C" int fb_tune(fb_ctx *ctx, int substeps, fb_tuning *best, double *ms_out)
{
  if (!ctx || substeps < 1) return FB_ERR_INVALID;
  if (!ctx->uploaded || (ctx->has_dust && !ctx->dust_uploaded)) return FB_ERR_STATE;
  KP &k = ctx->k;
  int rc = fb_profile(ctx, 1);
  if (rc) return rc;
  Snapshot sn;
  rc = snapshot_take(ctx, sn);
  if (rc) { snapshot_free(sn); fb_profile(ctx, 0); return rc; }
  const int cell_stages[] = {ST_POT, ST_SUB1, ST_VTERMS, ST_VUPDATE, ST_SUB2, ST_SUB3, ST_TVR};
  const int azi_stage[] = {ST_TAZI};
  const int rad_stage[] = {ST_TRAD};
  double total = 0.0;
  // 1. per-cell CTA width
  {
    const int cand[] = {64, 128, 256};
    int bestv = k.cell_bs;
    double bestms = 1e300;
    for (int c : cand) {
      k.cell_bs = c;
      const double ms = tune_measure(ctx, sn, substeps, cell_stages, 7);
      if (ms >= 0.0 && ms < bestms) { bestms = ms; bestv = c; }
    }
    k.cell_bs = bestv;
    total += bestms;
  }
  // 2. cells per thread and variant of the azimuthal pass
  {
    int bestv = k.azi_E, bestvar = k.azi_variant;
    double bestms = 1e300;
    for (int E = 1; E <= 4; E++) {
      if (!fb_azi_E_valid(k.ns, k.energy, E)) continue;
      for (int var = 1; var <= 8; var++) {
        if (fb_azi_variant(k.ns, k.energy, E, var) != var) continue;
        k.azi_E = E;
        k.azi_variant = var;
        const double ms = tune_measure(ctx, sn, substeps, azi_stage, 1);
        if (ms >= 0.0 && ms < bestms) { bestms = ms; bestv = E; bestvar = var; }
      }
    }
    k.azi_E = bestv;
    k.azi_variant = bestvar;
    total += bestms;
  }
  // 3. columns x rings per CTA of the radial pass
  {
    const int txs[] = {32, 64, 128};
    int btx = k.rad_tx, bch = k.rad_chunk;
    double bestms = 1e300;
    for (int tx : txs) {
      // powers of two and the chunks that fill whole waves of this width
      int chunks[10] = {4, 8, 16, 32};
      int nch = 4 + fb_rad_chunks_balanced(k, tx, chunks + 4, 6);
      for (int q = 0; q < nch; q++) {
        const int ch = chunks[q];
        bool seen = false;
        for (int u = 0; u < q; u++) seen = seen || (chunks[u] == ch);
        if (seen || ch > k.nr) continue;
        k.rad_tx = tx;
        k.rad_chunk = ch;
        const double ms = tune_measure(ctx, sn, substeps, rad_stage, 1);
        if (ms >= 0.0 && ms < bestms) { bestms = ms; btx = tx; bch = ch; }
      }
    }
    k.rad_tx = btx;
    k.rad_chunk = bch;
    total += bestms;
  }
  rc = snapshot_restore(ctx, sn);
  if (!rc) rc = (cudaStreamSynchronize(ctx->st) == cudaSuccess) ? FB_OK : FB_ERR_CUDA;
  snapshot_free(sn);
  fb_profile(ctx, 0);
  invalidate_graph(ctx);
  if (best) fb_get_tuning(ctx, best);
  if (ms_out) *ms_out = total;
  return rc;
}
