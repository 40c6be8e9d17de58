// fb_gas.cu -- FP64 kernels of one gas substep of AlgoGas
// (src/SourceEuler.c:398-716) for sm_100a.
//
// Every kernel restates the reference expression it replaces with the same
// operand order (the library is built with --fmad=false so that no multiply
// is fused into an add), citing the reference file:line.  Ring reductions
// (azimuthal means) use a fixed tree order inside one CTA: deterministic,
// but rounded differently from the reference's sequential sums (~1e-16
// relative).  Their algorithmic traffic is a few fields of 8 B per cell;
// the transport passes carry enough FP64 work per cell (IEEE divisions in
// every van Leer slope) that instruction issue, not HBM, bounds them.
#include <cuda_runtime.h>
#include <math.h>
#include "fb_dev.cuh"

int fb_pdl = 1;

#define FB_BS 256
#define FB_BS2 256  // most threads per CTA of the per-cell kernels (k.cell_bs <= FB_BS2)
#define RING_U 6    // cells per thread and batch of k_soundspeed

// per-cell kernels: blockIdx.y = ring, 128 consecutive azimuths per CTA
// per-cell kernels: CTAs of k.cell_bs azimuths (a ring segment) times rings
static inline dim3 grid2d(const KP &k, int rings) { return dim3((k.ns + k.cell_bs - 1) / k.cell_bs, rings); }

static __device__ __forceinline__ double min2(double a, double b) { return (b < a) ? b : a; }  // SourceEuler.c:293
static __device__ __forceinline__ double max2(double a, double b) { return (b > a) ? b : a; }  // SourceEuler.c:300

static __device__ __forceinline__ double dt_of(const KP &k, double dtov) { return dtov > 0.0 ? dtov : k.ctl->dt; }

// ------------------------------------------------------------ reductions
template <int BS>
static __device__ double block_sum(double v, double *sh)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (lane < BS / 32) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[0] = v;
  }
  __syncthreads();
  double r = sh[0];
  __syncthreads();
  return r;
}

static __device__ __forceinline__ double nu_ring(const KP &k, int i)
{
  // FViscosity(Rmed[i]) (Viscosity.c:23-69) for the supported laws:
  // ALPHAVISCOSITY*GLOBAL_SoundSpeed[i]^2*pow(r,1.5), or VISCOSITY.
  if (k.visc_mode == 1) return k.alpha * k.gcs[i] * k.gcs[i] * k.p15[i];
  if (k.visc_mode == 2) return k.nu_const;
  return 0.0;
}

// Sums of NV values over a CTA of any multiple of 32 threads (<= 1024);
// every thread gets the totals.  sh holds NV * 32 doubles.
template <int NV>
static __device__ void block_sums(double (&v)[NV], double *sh)
{
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) sh[q * 32 + w] = v[q];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < NV; q++) {
      double x = (lane < nw) ? sh[q * 32 + lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) sh[q * 32] = x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; q++) v[q] = sh[q * 32];
  __syncthreads();
}

static __device__ double block_min_dyn(double v, double *sh)
{
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    const double u = __shfl_down_sync(0xffffffffu, v, o);
    v = (u < v) ? u : v;
  }
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (lane < nw) ? sh[lane] : 1e300;
    for (int o = 16; o > 0; o >>= 1) {
      const double u = __shfl_down_sync(0xffffffffu, v, o);
      v = (u < v) ? u : v;
    }
    if (lane == 0) sh[0] = v;
  }
  __syncthreads();
  const double r = sh[0];
  __syncthreads();
  return r;
}

static __device__ void controller_body(const KP &k, double *sh, fb_ctl *c);
static __device__ void planet_prelude(const KP &k, fb_ctl *c);
// Work arrays of the planets' step.  k_planets is one thread and keeps them
// in shared memory: with them as local arrays of the thread, the device
// compiler of this toolkit produced stage derivatives whose x component read
// the distance array instead of the positions (found by comparing one step
// of a free planet with the reference's; the shared-memory form matches it
// to the last bit).
struct RkWork {
  double k[6][4 * FB_MAX_PLANETS];
  double dist[FB_MAX_PLANETS];
  double q0[4 * FB_MAX_PLANETS], q1[4 * FB_MAX_PLANETS], masses[FB_MAX_PLANETS];
};

static __device__ void rk5(const double *q0, double dt, const double *masses, double *q1, int n,
                           const int *feelothers, int indirect, RkWork &w);

// ---------------------------------------------------------------- CFL
// ConditionCFL (SourceEuler.c:1304-1552): one CTA per ring computes the
// azimuthal mean Vmoy[i] and the smallest per-cell limit of the ring; the
// controller takes the minimum over rings, adds the shear limit and returns
// ceil(deltaT/newdt).  DetectCrash (SourceEuler.c:51-69) rides along.
// One pass over the ring: the values each cell needs after the ring sums
// (the mean azimuthal velocity the CFL limits need) are kept in shared
// memory (3 nsec doubles), so a ring's CTA of up to 256 threads fits in 64
// registers a thread: four CTAs share an SM and a 512-ring grid runs in one
// wave.
#define CFL_BS 256
static inline int cfl_threads(int ns)
{
  const int t = ((ns + 3) / 4 + 31) / 32 * 32;
  return t < CFL_BS ? t : CFL_BS;
}
__global__ void __launch_bounds__(CFL_BS, 4) k_cfl(KP k)
{
  fb_grid_dependency();
  __shared__ double sh[6 * 32];
  extern __shared__ double cfl_sm[];
  const int i = blockIdx.x, ns = k.ns, T = blockDim.x, tid = threadIdx.x;
  const size_t base = (size_t)i * ns;
  const double *vt = k.vt + base, *vr = k.vr + base, *rho = k.rho + base;
  const bool cfl = (i >= 1);  // ConditionCFL's rings: One_or_active..Max_or_active-1
  if (i == 0 && tid == 0) planet_prelude(k, k.ctl);
  const double rmi = k.rmed[i], surf = k.surf[i], rs = k.indirect_smoothing;
#if FB_FAST
  // fast build: every cell of the ring lies rmed[i] from the star, so the
  // smoothed 1/d^3 of the star's sums is the ring's (within a few ulp of
  // the reference's per-cell value): one root and two divisions per ring
  const double dist2_ring = rmi * rmi + rs * rs;
  const double invd3_ring = 1.0 / dist2_ring / sqrt(dist2_ring);
#endif
  // ring sums: vtheta; ComputeForce (Force.c:77-253) for the star (x = y = 0,
  // mass 0) with rsmoothing = INDIRECTTERMSMOOTHING (SourceEuler.c:482);
  // GasTotalMass (SideEuler.c:15) and the barycentre sums (SideEuler.c:42-89)
  double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  // ConditionCFL's per-cell limits (SourceEuler.c:1390-1485): all but the
  // residual-velocity one are known before the ring mean; the sum under the
  // square root is evaluated in the reference's order once it is
  double *vtc = cfl_sm, *s12 = cfl_sm + ns, *s4 = cfl_sm + 2 * ns;
  const double dxrad = k.dxrad[i], dxtheta = k.dxtheta_cfl[i];
  // the quotients by the ring's constant lengths, each correctly rounded
  // through one reciprocal per ring
  const double dxmin = min2(dxrad, dxtheta);
  const double rdxmin = 1.0 / dxmin, rdxrad = 1.0 / dxrad, rdxtheta = 1.0 / dxtheta;
  int negd = 0, nege = 0, bad = 0;
  for (int j = tid; j < ns; j += T) {
    const double vtj = vt[j], vrj = vr[j], dens = rho[j];
    v[0] += vtj;
    if (dens < 0.0) negd = 1;
    if (!isfinite(dens) || !isfinite(vtj) || !isfinite(vrj)) bad = 1;
    if (k.energy) {
      const double en = k.e[base + j];
      if (en < 0.0) nege = 1;
      if (!isfinite(en)) bad = 1;
    }
    const double xc = rmi * k.cosaz[j];
    const double yc = rmi * k.sinaz[j];
    const double cellmass = surf * dens;
    const double dx = xc - 0.0, dy = yc - 0.0;
#if FB_FAST
    const double InvDist3 = invd3_ring;
#else
    const double d2 = dx * dx + dy * dy;
    const double dist2 = d2 + rs * rs;
    const double distance = sqrt(dist2);
    const double InvDist3 = 1.0 / dist2 / distance;
#endif
    v[1] += FB_G * cellmass * dx * InvDist3 * 1.0;
    v[2] += FB_G * cellmass * dy * InvDist3 * 1.0;
    v[3] += surf * dens;
    v[4] += surf * dens * xc;
    v[5] += surf * dens * yc;
    if (cfl) {
      const int jp = (j == ns - 1) ? 0 : j + 1;
      double invdt1 = fb_quot(k.cs[base + j], dxmin, rdxmin);
      double invdt2 = fb_quot(fabs(vrj), dxrad, rdxrad);
      double dvr = vr[ns + j] - vrj;
      double dvt = vt[jp] - vtj;
      if (dvr >= 0.0) dvr = 1e-10; else dvr = -dvr;
      if (dvt >= 0.0) dvt = 1e-10; else dvt = -dvt;
      double invdt4 = max2(fb_quot(dvr, dxrad, rdxrad), fb_quot(dvt, dxtheta, rdxtheta));
      invdt4 *= 4.0 * FB_CVNR * FB_CVNR;
      vtc[j] = vtj;
      s12[j] = invdt1 * invdt1 + invdt2 * invdt2;
      s4[j] = invdt4 * invdt4;
    }
  }
  block_sums<6>(v, sh);
  const double vmoy = v[0] / (double)ns;
  if (tid == 0) {
    k.vmoy[i] = vmoy;
    double *pp = k.partials + (size_t)i * 5;  // summed by the controller in ring order
    for (int q = 0; q < 5; q++) pp[q] = v[1 + q];
  }
  negd = __syncthreads_or(negd);
  nege = __syncthreads_or(nege);
  bad = __syncthreads_or(bad);
  if (tid == 0) {
    if (negd) atomicOr(&k.ctl->neg_dens_flag, 1);
    if (nege) atomicOr(&k.ctl->neg_energy_flag, 1);
    if (bad) atomicOr(&k.ctl->nonfinite, 1);
  }
  if (cfl) {
    const double viscosity = nu_ring(k, i);
    const double invdt5 = (viscosity != 0.0) ? viscosity * 4.0 / k.mindx2[i] : 1e-10;
    // thermal diffusion's limit (SourceEuler.c:1411-1428): entropy
    // diffusion's per ring; explicit radiative diffusion's per cell (below),
    // which replaces it when both are on
    const double invdt6_ring = (k.energy && k.ent_diff) ? k.diffusivity * 4.0 / k.mindx2[i] : 1e-10;
    // the ring's limit is the smallest CFLSECURITY / sqrt(S) over its cells;
    // a correctly rounded square root and quotient are monotone, so it is
    // the limit of the largest S, to the last bit: one root and one division
    // per ring.  A NaN sum is skipped as the reference's `dt < newdt` skips
    // it; S >= invdt5^2 >= 1e-20 otherwise.
    double smax = -1.0;
    for (int j = tid; j < ns; j += T) {  // each thread reads back its own cells
      double vres = k.fast_transport ? vtc[j] - vmoy : vtc[j];
      double invdt3 = fb_quot(fabs(vres), dxtheta, rdxtheta);
      double invdt6 = invdt6_ring;
      if (k.energy && k.rad_diff == 1) invdt6 = k.td_rad[base + j];  // k_td_cfl, just before this kernel
      const double S = s12[j] + invdt3 * invdt3 + s4[j] + invdt5 * invdt5 + invdt6 * invdt6;
      if (S > smax) smax = S;
    }
    smax = -block_min_dyn(-smax, sh);
    if (tid == 0) k.ringmin[i] = (smax > 0.0) ? FB_CFLSECURITY / sqrt(smax) : 1e30;
  }
  // the last CTA to finish runs the controller (no waiting: whoever comes
  // last sees every other ring's results)
  __shared__ int last;
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    last = (atomicAdd(&k.ctl->cfl_done, 1u) == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ fb_ctl cs;
  unsigned long long *dst = (unsigned long long *)&cs;
  const unsigned long long *src = (const unsigned long long *)k.ctl;
  for (int w = tid; w < (int)(sizeof(fb_ctl) / 8); w += T) dst[w] = __ldcg(src + w);
  __syncthreads();
  controller_body(k, sh, &cs);
  __syncthreads();
  if (tid == 0) cs.cfl_done = 0;
  __syncthreads();
  unsigned long long *out = (unsigned long long *)k.ctl;
  for (int w = tid; w < (int)(sizeof(fb_ctl) / 8); w += T) out[w] = dst[w];
}

void fb_launch_cfl(const KP &k, cudaStream_t s)
{
  fb_launch(k_cfl, k.nr, cfl_threads(k.ns), 3 * (size_t)k.ns * sizeof(double), s, k);
}

// The planets' step of the substep, after the controller has set dt:
// AdvanceSystemRK5 (Pframeforce.c:163-266) and RotatePsys (Psys.c:352-372).
// One thread.  No other kernel of the substep reads the positions before the
// particles' velocity update, so this kernel runs on a branch of its own
// beside the gas kernels; with particles it also evaluates the planet terms
// of UpdateDustVelocities (DustUpdate.c:342-352) at the new positions.
__global__ void k_planets(KP k, fb_dust_ctl *dc, double thick, double aspect, double flaring)
{
  fb_grid_dependency();
  fb_ctl *c = k.ctl;
  c->domega = 0.0;
  if (c->status != FB_OK) return;
  const int np = c->np;
  const double dt = c->dt;
  // corotating frame: GetPsysInfo(sys, MARK) (SourceEuler.c:476, Psys.c:
  // 323-326): the first planet's position at the start of the substep
  const double xmark = (np > 0) ? c->px[0] : 0.0, ymark = (np > 0) ? c->py[0] : 0.0;
  // AdvanceSystemRK5 (Pframeforce.c:163-266)
  if (!k.forced_circular) {
    __shared__ RkWork rw;
    double *q0 = rw.q0, *q1 = rw.q1, *masses = rw.masses;
    for (int i = 0; i < np; i++) {
      q0[i] = c->px[i]; q0[i + np] = c->py[i]; q0[i + 2 * np] = c->pvx[i]; q0[i + 3 * np] = c->pvy[i];
      masses[i] = c->pm[i];
    }
    if (np > 0) rk5(q0, dt, masses, q1, np, c->pfeelothers, k.indirect_term, rw);
    for (int i = 0; i < np; i++) {
      c->px[i] = q1[i]; c->py[i] = q1[i + np]; c->pvx[i] = q1[i + 2 * np]; c->pvy[i] = q1[i + 3 * np];
    }
  } else {
    for (int i = 0; i < np; i++) {
      double x = c->px[i], y = c->py[i];
      double theta = atan2(y, x);
      double vx = c->pvx[i], vy = c->pvy[i];
      double r = sqrt(x * x + y * y);
      double v = sqrt(vx * vx + vy * vy);
      double omega = (-y * vx + x * vy) / r / r;
      double dtheta = omega * dt;
      c->px[i] = r * cos(theta + dtheta);
      c->py[i] = r * sin(theta + dtheta);
      c->pvx[i] = -v * sin(theta + dtheta);
      c->pvy[i] = v * cos(theta + dtheta);
    }
  }
  // corotating frame (SourceEuler.c:516-524): OmegaFrame becomes the angle
  // the first planet turned through during the step (GetPsysInfo GET,
  // Psys.c:327-337) over dt; CorrectVtheta follows with the change
  if (k.corot && np > 0) {
    const double x = c->px[0], y = c->py[0];
    const double d2 = sqrt(x * x + y * y);
    const double d1 = sqrt(xmark * xmark + ymark * ymark);
    const double cross = xmark * y - x * ymark;
    const double omega_new = asin(cross / (d1 * d2)) / dt;
    c->domega = omega_new - c->omega_frame;
    c->omega_frame = omega_new;
  }
  // RotatePsys (Psys.c:352-372) with angle OmegaFrame*dt
  {
    double angle = c->omega_frame * dt;
    double sint = sin(angle), cost = cos(angle);
    for (int i = 0; i < np; i++) {
      double xt = c->px[i], yt = c->py[i];
      c->px[i] = xt * cost + yt * sint;
      c->py[i] = -xt * sint + yt * cost;
      xt = c->pvx[i]; yt = c->pvy[i];
      c->pvx[i] = xt * cost + yt * sint;
      c->pvy[i] = -xt * sint + yt * cost;
    }
  }
  if (dc) {
    for (int p = 0; p < np; p++) {
      const double xp = c->px[p], yp = c->py[p];
      const double rpl = sqrt(xp * xp + yp * yp);
      dc->pl_r[p] = rpl;
      dc->pl_t[p] = atan2(yp, xp);
      dc->pl_eps[p] = thick * aspect * pow(0.5 * rpl, 1.0 + flaring) * pow(2.0, 1.0 + flaring);
    }
  }
}

// CorrectVtheta (SideEuler.c:1133-1147): vtheta -= domega Rmed on rings
// 0..nr-1 after the frame's angular velocity changed by domega
__global__ void __launch_bounds__(FB_BS2) k_correct_vtheta(KP k)
{
  fb_grid_dependency();
  const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k.ns) return;
  const double domega = k.ctl->domega;
  k.vt[(size_t)i * k.ns + j] -= domega * k.rmed[i];
}

void fb_launch_correct_vtheta(const KP &k, cudaStream_t s)
{
  fb_launch(k_correct_vtheta, grid2d(k, k.nr), k.cell_bs, 0, s, k);
}

void fb_launch_planets(const KP &k, const PP *pp, cudaStream_t s)
{
  if (pp && pp->feel_planets)
    fb_launch(k_planets, 1, 1, 0, s, k, pp->dc, pp->thicksmoothing, pp->aspectratio, pp->flaringindex);
  else
    fb_launch(k_planets, 1, 1, 0, s, k, nullptr, 0.0, 0.0, 0.0);
}

// ------------------------------------------------------------ controller
static __device__ double dev_aspect_ratio(const KP &k, double rad)
{
  // AspectRatio (Viscosity.c:107-123) with TRANSITION* at their defaults
  double aspectratio = k.aspectratio;
  double rmin = 0.0 - 1.0 * k.aspectratio, rmax = 0.0 + 1.0 * k.aspectratio;
  if ((rad >= rmin) && (rad <= rmax)) aspectratio *= exp((rmax - rad) / (rmax - rmin) * log(1.0));
  return aspectratio;
}

// DerivMotionRK5 (RungeKunta.c:13-53)
static __device__ void rk5_deriv(const double *q, const double *masses, double *deriv, int n,
                                 double dt, const int *feelothers, int indirect, double *Dist)
{
  const double *x = q, *y = q + n, *vx = q + 2 * n, *vy = q + 3 * n;
  double *dx = deriv, *dy = deriv + n, *dvx = deriv + 2 * n, *dvy = deriv + 3 * n;
  for (int i = 0; i < n; i++) Dist[i] = sqrt(x[i] * x[i] + y[i] * y[i]);
  for (int i = 0; i < n; i++) {
    dx[i] = vx[i];
    dy[i] = vy[i];
    dvx[i] = -FB_G * 1.0 / Dist[i] / Dist[i] / Dist[i] * x[i];
    dvy[i] = -FB_G * 1.0 / Dist[i] / Dist[i] / Dist[i] * y[i];
    for (int j = 0; j < n; j++) {
      if (indirect) {
        dvx[i] -= FB_G * masses[j] / Dist[j] / Dist[j] / Dist[j] * x[j];
        dvy[i] -= FB_G * masses[j] / Dist[j] / Dist[j] / Dist[j] * y[j];
      }
      if ((j != i) && feelothers[i]) {
        double dist = (x[i] - x[j]) * (x[i] - x[j]) + (y[i] - y[j]) * (y[i] - y[j]);
        dist = sqrt(dist);
        dvx[i] += FB_G * masses[j] / dist / dist / dist * (x[j] - x[i]);
        dvy[i] += FB_G * masses[j] / dist / dist / dist * (y[j] - y[i]);
      }
    }
  }
  for (int i = 0; i < 4 * n; i++) deriv[i] *= dt;
}

// RungeKunta (RungeKunta.c:64-91)
static __device__ void rk5(const double *q0, double dt, const double *masses, double *q1, int n,
                           const int *feelothers, int indirect, RkWork &w)
{
  // k2..k5 enter the first translations multiplied by 0.0; the reference
  // seeds them with the previous call's k6 (RungeKunta.c:73-75), which is
  // finite, so zeros give the same sums.
  double *k1 = w.k[0], *k2 = w.k[1], *k3 = w.k[2], *k4 = w.k[3], *k5 = w.k[4], *k6 = w.k[5];
  for (int s = 0; s < 6; s++)
    for (int i = 0; i < 4 * FB_MAX_PLANETS; i++) w.k[s][i] = 0.0;
  double *Dist = w.dist;
  const int m = 4 * n;
  rk5_deriv(q0, masses, k1, n, dt, feelothers, indirect, Dist);
  for (int i = 0; i < m; i++) q1[i] = q0[i] + 0.2 * k1[i] + 0.0 * k2[i] + 0.0 * k3[i] + 0.0 * k4[i] + 0.0 * k5[i];
  rk5_deriv(q1, masses, k2, n, dt, feelothers, indirect, Dist);
  for (int i = 0; i < m; i++) q1[i] = q0[i] + 0.075 * k1[i] + 0.225 * k2[i] + 0.0 * k3[i] + 0.0 * k4[i] + 0.0 * k5[i];
  rk5_deriv(q1, masses, k3, n, dt, feelothers, indirect, Dist);
  for (int i = 0; i < m; i++) q1[i] = q0[i] + 0.3 * k1[i] + -0.9 * k2[i] + 1.2 * k3[i] + 0.0 * k4[i] + 0.0 * k5[i];
  rk5_deriv(q1, masses, k4, n, dt, feelothers, indirect, Dist);
  for (int i = 0; i < m; i++)
    q1[i] = q0[i] + -11.0 / 54.0 * k1[i] + 2.5 * k2[i] + -70.0 / 27.0 * k3[i] + 35.0 / 27.0 * k4[i] + 0.0 * k5[i];
  rk5_deriv(q1, masses, k5, n, dt, feelothers, indirect, Dist);
  for (int i = 0; i < m; i++)
    q1[i] = q0[i] + 1631.0 / 55296.0 * k1[i] + 175.0 / 512.0 * k2[i] + 575.0 / 13824.0 * k3[i] +
            44275.0 / 110592.0 * k4[i] + 253.0 / 4096.0 * k5[i];
  rk5_deriv(q1, masses, k6, n, dt, feelothers, indirect, Dist);
  for (int i = 0; i < m; i++)
    q1[i] = q0[i] + 37.0 / 378.0 * k1[i] + 250.0 / 621.0 * k3[i] + 125.0 / 594.0 * k4[i] + 512.0 / 1771.0 * k6[i];
}

// The scalar part of one substep of AlgoGas, SourceEuler.c:398-531, run by
// the last CTA of k_cfl: its threads reduce the per-ring CFL limits, the
// shear limits and the force partials (fixed tree order), then thread 0 runs
// the scalar logic on a shared-memory copy of the control block.
// The planet terms of the substep that do not depend on its time step:
// masses (SourceEuler.c:402-418), the n-body limit (SourceEuler.c:421-440)
// and FillForcesArrays' planet parameters at the current positions
// (Pframeforce.c:44-90).  Run by one thread of CTA 0 of the CFL kernel while
// the other CTAs work on their rings; the controller (last CTA) reads them.
static __device__ void planet_prelude(const KP &k, fb_ctl *c)
{
  const int np = c->np;
  if (k.masstaper > 1e-2) {
    double mt = (c->physical_time - c->physical_time_initial) / (k.masstaper * 2.0 * M_PI);
    mt = (mt > 1.0 ? 1.0 : pow(sin(mt * M_PI / 2.0), 2.0));
    if (mt < 1.0)
      for (int p = 0; p < np; p++) c->pm[p] = c->pinit[p] + (c->pfinal[p] - c->pinit[p]) * mt;
  } else {
    for (int p = 0; p < np; p++)
      if (c->pacc[p] < 1e-10) c->pm[p] = c->pfinal[p];
  }
  double dtnbody;
  if (np > 1) {
    dtnbody = 1e5;
    for (int a = 0; a < np; a++)
      for (int b = a + 1; b < np; b++) {
        double xk = c->px[a], xj = c->px[b], yk = c->py[a], yj = c->py[b];
        double mk = c->pm[a], mj = c->pm[b];
        double dist = sqrt((xk - xj) * (xk - xj) + (yk - yj) * (yk - yj));
        double buf = 2.0 * M_PI * sqrt(dist * dist * dist / (mk + mj + 1e-8)) / FB_BINARYSECURITY;
        dtnbody = min2(dtnbody, buf);
      }
  } else {
    dtnbody = 100.0;
  }
  c->dtnbody = dtnbody;
  double planetmass_taper = 1.0;
  if (k.masstaper > 1e-2) {
    double mt = (c->physical_time - c->physical_time_initial) / (k.masstaper * 2.0 * M_PI);
    planetmass_taper = (mt > 1.0 ? 1.0 : .5 * (1.0 - cos(M_PI * mt)));
  }
  for (int p = 0; p < np; p++) {
    double xplanet = c->px[p], yplanet = c->py[p];
    double mplanet = c->pm[p] * planetmass_taper;
    double PlanetDistance = sqrt(xplanet * xplanet + yplanet * yplanet);
    double InvPlanetDistance3 = 1.0 / PlanetDistance / PlanetDistance / PlanetDistance;
    double smoothing;
    if (k.roche) {
      double RRoche = PlanetDistance * pow((1.0 / 3.0 * mplanet), 1.0 / 3.0);
      smoothing = RRoche * k.rochesmoothing;
    } else {
      smoothing = k.thicksmoothing * dev_aspect_ratio(k, PlanetDistance) * pow(PlanetDistance, 1.0 + k.flaringindex);
    }
    c->pot_m[p] = mplanet;
    c->pot_x[p] = xplanet;
    c->pot_y[p] = yplanet;
    c->pot_smooth2[p] = smoothing * smoothing;
    c->pot_invd3[p] = InvPlanetDistance3;
  }
}

static __device__ void controller_body(const KP &k, double *sh, fb_ctl *c)
{
  const int nr = k.nr, tid = threadIdx.x, T = blockDim.x;
  // ConditionCFL reduction (SourceEuler.c:1336-1497), the ring partials of
  // the forces and sums; every load is issued before the reductions
  double m = 1e30;
  double f[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int i = tid; i < nr; i += T) {
    const double rmin = (i >= 1) ? __ldcg(k.ringmin + i) : 1e30;
    const double v0 = __ldcg(k.vmoy + i);
    const double v1 = (i < nr - 1) ? __ldcg(k.vmoy + i + 1) : 0.0;
    const double *p = k.partials + (size_t)i * 5;
    for (int q = 0; q < 5; q++) f[q] += __ldcg(p + q);
    if (rmin < m) m = rmin;
    if (i < nr - 1) {
      double d = (k.pmax - k.pmin) * FB_CFLSECURITY / (double)k.ns /
                 fabs(v0 * k.invrmed[i] - v1 * k.invrmed[i + 1]);
      if (d < m) m = d;
    }
  }
  const double newdt_cells = block_min_dyn(m, sh);
  block_sums<5>(f, sh);
  if (tid != 0) return;
  const double dtnbody = c->dtnbody;  // planet_prelude
  // DetectCrash of the substep's starting state (SourceEuler.c:545-566):
  // Crashed is the energy test alone (it overwrites the density test's
  // result; an isothermal run's energy grid holds EnergyMed >= 0 and never
  // crashes).  The first crash's time is kept and its state copied by the
  // potential kernel of this substep, which runs before anything changes it.
  c->crash_snap_now = 0;
  if (c->neg_dens_flag) c->neg_dens_substeps += 1;
  if (k.energy && c->neg_energy_flag) {
    if (c->crashes == 0) {
      c->crash_time = c->physical_time;
      c->crash_snap_now = k.crash_snap ? 1 : 0;
      c->crash_snapped = c->crash_snap_now;
    }
    c->crashes += 1;
    c->crash_substeps += 1;
  }
  c->neg_dens_flag = 0;
  c->neg_energy_flag = 0;
  // ConditionCFL reduction (SourceEuler.c:1336-1497) and substep count
  const double deltaT = c->DT - c->dtemp;
  double newdt = newdt_cells;
  if (k.dust_min_ts) {  // SourceEuler.c:1501-1507
    double dt_fb = 0.5 * *k.dust_min_ts;
    if (dt_fb == 0.0) dt_fb = 1e10;
    if (dt_fb < newdt) newdt = dt_fb;
  }
  if (deltaT < newdt) newdt = deltaT;
  const double ncfl = ceil(deltaT / newdt);
  if (!(ncfl >= 1.0) || ncfl > 2.0e9) {
    c->status = FB_ERR_SUBSTEPS;
    c->done = 1;
    return;
  }
  const int gastimestepcfl = (int)ncfl;
  const double dthydro = (c->DT - c->dtemp) / (double)gastimestepcfl;
  const double dt = min2(dthydro, dtnbody);
  c->dthydro = dthydro;
  c->dt = dt;
  c->dtemp += dt;
  if (dt < c->mindt) c->mindt = dt;
  if (dt > c->maxdt) c->maxdt = dt;
  // DiskOnPrimaryAcceleration = ComputeAccel(...) (SourceEuler.c:482)
  const double fx = f[0], fy = f[1], mass = f[2], xb = f[3], yb = f[4];
  c->disk_acc_x = 0.0 + fx;
  c->disk_acc_y = 0.0 + fy;
  c->mdisc = mass;
  // ComputeOppositeAccelerationOfBarycenter (SideEuler.c:91-112)
  c->bary_x[2] = xb / (1.0 + mass);
  c->bary_y[2] = yb / (1.0 + mass);
  c->disk_acc_alt_x = -(c->bary_x[2] - 2.0 * c->bary_x[1] + c->bary_x[0]) / (dt * dt);
  c->disk_acc_alt_y = -(c->bary_y[2] - 2.0 * c->bary_y[1] + c->bary_y[0]) / (dt * dt);
  c->bary_x[0] = c->bary_x[1]; c->bary_x[1] = c->bary_x[2];
  c->bary_y[0] = c->bary_y[1]; c->bary_y[1] = c->bary_y[2];
  // FillForcesArrays prelude (Pframeforce.c:44-90): the indirect term (the
  // planets' parameters come from planet_prelude)
  c->ind_x = -c->disk_acc_x;
  c->ind_y = -c->disk_acc_y;
  if (k.alt_gas_it) { c->ind_x = -c->disk_acc_alt_x; c->ind_y = -c->disk_acc_alt_y; }
  if (!k.indirect_term) { c->ind_x = 0.0; c->ind_y = 0.0; }
  // AdvanceSystemRK5 and RotatePsys follow in k_planets, which runs beside
  // the next kernels of the substep
  c->t_sub = c->physical_time;  // what FillForcesArrays' turbulent potential sees
  c->physical_time += dt;  // SourceEuler.c:714 (no kernel in this substep reads it)
  c->substeps += 1;
  c->done = (c->dtemp < 0.999999999 * c->DT) ? 0 : 1;
  if (c->nonfinite) { c->status = FB_ERR_NAN; c->done = 1; }
}

// ------------------------------------------------------------ sound speed
// ComputeSoundSpeed (SourceEuler.c:2323-2343), energy equation, and the
// ring means GLOBAL_SoundSpeed that mpi_make1Dprofile (axilib.c:5-60) makes
// inside ComputeViscousTerms (Viscosity.c:247-248).
__global__ void __launch_bounds__(FB_BS) k_soundspeed(KP k, int update_gcs)
{
  fb_grid_dependency();
  __shared__ double sh[32];
  const int i = blockIdx.x, ns = k.ns;
  const size_t base = (size_t)i * ns;
  double s = 0.0;
  for (int j0 = threadIdx.x; j0 < ns; j0 += RING_U * FB_BS) {
    double ev[RING_U], dv[RING_U];
#pragma unroll
    for (int u = 0; u < RING_U; u++) {
      const int j = j0 + u * FB_BS;
      if (j < ns) {
        ev[u] = k.e[base + j];
        dv[u] = k.rho[base + j];
      }
    }
#pragma unroll
    for (int u = 0; u < RING_U; u++) {
      const int j = j0 + u * FB_BS;
      if (j < ns) {
        double c = sqrt(k.gamma * (k.gamma - 1.0) * ev[u] / dv[u]);
        k.cs[base + j] = c;
        s += c;
      }
    }
  }
  if (update_gcs) {
    s = block_sum<FB_BS>(s, sh);
    if (threadIdx.x == 0) k.gcs[i] = s / (double)ns;
  }
}

void fb_launch_soundspeed(const KP &k, int update_gcs, cudaStream_t s)
{
  fb_launch(k_soundspeed, k.nr, FB_BS, 0, s, k, update_gcs);
}

// ----------------------------------------------------------- potential
// FillForcesArrays (Pframeforce.c:44-129): star + planets + indirect terms.
__global__ void __launch_bounds__(FB_BS2) k_potential(KP k)
{
  fb_grid_dependency();
  const fb_ctl *c = k.ctl;
  const int np = c->np;
  const int use_ind = (!k.discard_gas_it) && (fabs(k.pmax - k.pmin - 2. * M_PI) < 0.01);
  {
    const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k.ns) return;
    const size_t l = (size_t)i * k.ns + j;
    const double x = k.rmed[i] * k.cosaz[j];
    const double y = k.rmed[i] * k.sinaz[j];
    double P = 0.0, IP = 0.0;
    for (int p = 0; p < np; p++) {
      const double xplanet = c->pot_x[p], yplanet = c->pot_y[p], mplanet = c->pot_m[p];
      double distance = (x - xplanet) * (x - xplanet) + (y - yplanet) * (y - yplanet);
      double distancesmooth = sqrt(distance + c->pot_smooth2[p]);
      double pot = -FB_G * mplanet / distancesmooth;
      if (k.indirect_term) {
        const double ind = FB_G * mplanet * c->pot_invd3[p] * (x * xplanet + y * yplanet);
        pot += ind;
        if (k.dust_feel_planets) IP = ind;  // Pframeforce.c:102-103 assigns, last planet wins
      }
      P += pot;
    }
    {
      const double InvDistance = k.invrmed[i];  // 1.0 / Rmed[i], correctly rounded on the host
      double pot = -FB_G * 1.0 * InvDistance;
      if (use_ind) {
        pot -= c->ind_x * x + c->ind_y * y;
        if (k.dust_feel_disk) IP -= c->ind_x * x + c->ind_y * y;
      }
      P += pot;
    }
    k.pot[l] = P;
    if (k.particles) k.indpot[l] = IP;  // IndPotential (Pframeforce.c:55-121)
    if (c->crash_snap_now) {  // the first crash's state (WriteDiskPolar ..., 999)
      const size_t n = (size_t)k.nr * k.ns;
      k.crash_snap[l] = k.rho[l];
      k.crash_snap[n + l] = k.vr[l];
      k.crash_snap[2 * n + l] = k.vt[l];
      if (k.energy) k.crash_snap[3 * n + l] = k.e[l];
    }
  }
}

void fb_launch_potential(const KP &k, cudaStream_t s)
{
  fb_launch(k_potential, grid2d(k, k.nr), k.cell_bs, 0, s, k);
}

// ------------------------------------------------------------ SubStep1
static __device__ __forceinline__ double pressure_at(const KP &k, size_t l)
{
  // ComputePressureField (SourceEuler.c:2414-2438)
  if (!k.energy) return k.rho[l] * k.cs[l] * k.cs[l];
  return (k.gamma - 1.0) * k.e[l];
}

// SubStep1 (SourceEuler.c:765-1009) without dust: pressure, potential and
// curvature terms into VradInt (i >= 1) and VthetaInt (all rings).  At most
// 64 registers, so that four 256-thread CTAs share an SM (68 would allow three).
__global__ void __launch_bounds__(FB_BS2, 4) k_substep1(KP k)
{
  fb_grid_dependency();
  const int ns = k.ns;
  const double dt = k.ctl->dt;
  const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j;
  const size_t ljm = (j == 0) ? (size_t)i * ns + ns - 1 : l - 1;
  const size_t ljp = (j == ns - 1) ? (size_t)i * ns : l + 1;
  const size_t lim = (i >= 1) ? l - ns : l;
  // every load first (the stores below could alias them for the compiler)
  const double Pl = pressure_at(k, l), Pjm = pressure_at(k, ljm);
  const double rl = k.rho[l], rjm = k.rho[ljm], potl = k.pot[l], potjm = k.pot[ljm], vtl = k.vt[l];
  const double invdxtheta = k.invdxtheta[i], torque = k.supp_torque[i];
  double Plim = 0.0, rlim = 0.0, potlim = 0.0, vtjp = 0.0, vtlim = 0.0, vtjplim = 0.0, vrl = 0.0;
  double invdiffrmed = 0.0, rinf = 0.0, invrinf = 0.0;
  if (i >= 1) {
    Plim = pressure_at(k, lim);
    rlim = k.rho[lim];
    potlim = k.pot[lim];
    vtjp = k.vt[ljp];
    vtlim = k.vt[lim];
    vtjplim = k.vt[ljp - ns];
    vrl = k.vr[l];
    invdiffrmed = k.invdiffrmed[i];
    rinf = k.rinf[i];
    invrinf = k.invrinf[i];
  }
  double ipl = 0.0, iplim = 0.0, ipjm = 0.0;
  if (k.particles) {
    ipl = k.indpot[l];
    ipjm = k.indpot[ljm];
    if (i >= 1) iplim = k.indpot[lim];
  }
  k.pres[l] = Pl;
  if (i >= 1) {
    double gradp = (Pl - Plim) * 2.0 / (rl + rlim) * invdiffrmed;
    double gradphi = (potl - potlim) * invdiffrmed;
    double vt2 = vtl + vtjp + vtlim + vtjplim;
    vt2 = vt2 / 4.0 + rinf * omf(k);
    vt2 = vt2 * vt2;
    k.vri[l] = vrl + dt * (-gradp - gradphi + vt2 * invrinf);
    if (k.particles) {  // RadGradP, RadIndAcc (SourceEuler.c:875-877)
      k.rgp[l] = (Pl - Plim) * invdiffrmed;
      k.rind[l] = -(ipl - iplim) * invdiffrmed;
    }
  }
  {
    double gradp = (Pl - Pjm) * 2.0 / (rl + rjm) * invdxtheta;
    double gradphi = (potl - potjm) * invdxtheta;
    double vti = vtl - dt * (gradp + gradphi);
    vti += dt * torque;
    k.vti[l] = vti;
    if (k.particles) {  // AziGradP, AziIndAcc (SourceEuler.c:944-951)
      k.agp[l] = (Pl - Pjm) * invdxtheta;
      k.aind[l] = -(ipl - ipjm) * invdxtheta;
    }
  }
}

void fb_launch_substep1(const KP &k, cudaStream_t s)
{
  fb_launch(k_substep1, grid2d(k, k.nr), k.cell_bs, 0, s, k);
}

// ------------------------------------------------------- viscous stresses
// ComputeViscousTerms (Viscosity.c:159-303) incl. ComputeDivergenceVelocity
// (SourceEuler.c:2373-2412) at cell (i, j): DivV, TAUrr, TAUpp (all rings),
// TAUrp (i >= 1); taus = 0: DivV alone.
struct Stress {
  double div, trr, tpp, trp;
};
static __device__ __forceinline__ Stress stress_at(const KP &k, const double *__restrict__ vr,
                                                   const double *__restrict__ vt, int i, int j, bool taus)
{
  const int ns = k.ns;
  const double invdphi = k.invdphi, onethird = 1.0 / 3.0;
  const size_t l = (size_t)i * ns + j;
  const size_t lip = l + ns;
  const size_t ljp = (j == ns - 1) ? (size_t)i * ns : l + 1;
  const size_t ljm = (j == 0) ? (size_t)i * ns + ns - 1 : l - 1;
  // every load first
  const double vrl = vr[l], vrip = vr[lip], vtl = vt[l], vtjp = vt[ljp];
  const double rsup = k.rsup[i], rinf = k.rinf[i], invdiffrsup = k.invdiffrsup[i], invrmed = k.invrmed[i];
  double rl = 0.0, vtim = 0.0, vrjm = 0.0, rim = 0.0, rjm = 0.0, rjmim = 0.0, invrmedm = 0.0, invdiffrmed = 0.0,
         invrinf = 0.0;
  if (taus) {
    rl = k.rho[l];
    if (i >= 1) {
      const size_t lim = l - ns, ljmim = ljm - ns;
      vtim = vt[lim];
      vrjm = vr[ljm];
      rim = k.rho[lim];
      rjm = k.rho[ljm];
      rjmim = k.rho[ljmim];
      invrmedm = k.invrmed[i - 1];
      invdiffrmed = k.invdiffrmed[i];
      invrinf = k.invrinf[i];
    }
  }
  Stress st;
  double div = (vrip * rsup - vrl * rinf) * invdiffrsup * invrmed;
  div += (vtjp - vtl) * invdphi * invrmed;
  st.div = div;
  st.trr = st.tpp = st.trp = 0.0;
  if (taus) {
    const double Drr = (vrip - vrl) * invdiffrsup;
    const double Dpp = (vtjp - vtl) * invdphi * invrmed + 0.5 * (vrip + vrl) * invrmed;
    const double viscosity = nu_ring(k, i);
    st.trr = 2.0 * rl * viscosity * (Drr - onethird * div);
    st.tpp = 2.0 * rl * viscosity * (Dpp - onethird * div);
    if (i >= 1) {
      const double Drp = 0.5 * (rinf * (vtl * invrmed - vtim * invrmedm) * invdiffrmed + (vrl - vrjm) * invdphi * invrinf);
      st.trp = 2.0 * 0.25 * (rl + rim + rjm + rjmim) * viscosity * Drp;
    }
  }
  return st;
}

__global__ void __launch_bounds__(FB_BS2) k_viscous_terms(KP k, const double *__restrict__ vr,
                                                         const double *__restrict__ vt)
{
  fb_grid_dependency();
  const int ns = k.ns;
  const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j;
  const Stress st = stress_at(k, vr, vt, i, j, true);
  k.divv[l] = st.div;
  k.trr[l] = st.trr;
  k.tpp[l] = st.tpp;
  if (i >= 1) k.trp[l] = st.trp;
}

void fb_launch_viscous_terms(const KP &k, const double *vr, const double *vt, cudaStream_t s)
{
  fb_launch(k_viscous_terms, grid2d(k, k.nr), k.cell_bs, 0, s, k, vr, vt);
}

// UpdateVelocitiesWithViscosity (Viscosity.c:305-378)
__global__ void __launch_bounds__(FB_BS2) k_viscous_update(KP k, double *vr, double *vt, double dtov)
{
  fb_grid_dependency();
  const int ns = k.ns, nr = k.nr;
  const double DeltaT = dt_of(k, dtov), invdphi = k.invdphi;
  const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j;
  if (i < 1) return;
  const size_t ljp = (j == ns - 1) ? (size_t)i * ns : l + 1;
  const size_t ljm = (j == 0) ? (size_t)i * ns + ns - 1 : l - 1;
  const size_t lim = l - ns, lip = l + ns;
  // every load first
  const double trpl = k.trp[l], trpip = k.trp[lip], trpjp = k.trp[ljp];
  const double tppl = k.tpp[l], tppjm = k.tpp[ljm], tppim = k.tpp[lim];
  const double trrl = k.trr[l], trrim = k.trr[lim];
  const double rl = k.rho[l], rjm = k.rho[ljm], rim = k.rho[lim];
  const double vtl = vt[l], vrl = vr[l];
  const double invrmed = k.invrmed[i], rsup = k.rsup[i], rinf = k.rinf[i], invdiffrsup = k.invdiffrsup[i];
  const double invrinf = k.invrinf[i], rmed = k.rmed[i], rmedm = k.rmed[i - 1], invdiffrmed = k.invdiffrmed[i];
  if (i < nr - 1) {
    vt[l] = vtl + DeltaT * invrmed *
                      ((rsup * trpip - rinf * trpl) * invdiffrsup + (tppl - tppjm) * invdphi + 0.5 * (trpl + trpip)) /
                      (0.5 * (rl + rjm));
  }
  vr[l] = vrl + DeltaT * invrinf *
                    ((rmed * trrl - rmedm * trrim) * invdiffrmed + (trpjp - trpl) * invdphi - 0.5 * (tppl + tppim)) /
                    (0.5 * (rl + rim));
}

void fb_launch_viscous_update(const KP &k, double *vr, double *vt, double dt_override, cudaStream_t s)
{
  fb_launch(k_viscous_update, grid2d(k, k.nr), k.cell_bs, 0, s, k, vr, vt, dt_override);
}

// ------------------------------------------------------------ SubStep2
// SubStep2 (SourceEuler.c:1012-1116) followed by the copies of
// SourceEuler.c:617-622: artificial viscosity from VradInt/VthetaInt into
// Vrad/Vtheta (and EnergyInt into Energy).  Rings the reference never
// writes in VradNew/VthetaNew/EnergyInt (ring 0 and ring nr of VradNew, ring
// nr of the others) are zero, and the copies spread those zeros.
static __device__ __forceinline__ double q_r(const KP &k, size_t l, size_t lip)
{
  double dv = k.vri[lip] - k.vri[l];
  return (dv < 0.0) ? FB_CVNR * FB_CVNR * k.rho[l] * dv * dv : 0.0;
}
static __device__ __forceinline__ double q_t(const KP &k, size_t l, size_t ljp)
{
  double dv = k.vti[ljp] - k.vti[l];
  return (dv < 0.0) ? FB_CVNR * FB_CVNR * k.rho[l] * dv * dv : 0.0;
}

// At most 48 registers: five 256-thread CTAs per SM (SubStep2 20.6 -> 19.0 us;
// the same cap made the stress kernels and SubStep3 slower).
__global__ void __launch_bounds__(FB_BS2, 5) k_substep2(KP k)
{
  fb_grid_dependency();
  const int ns = k.ns, nr = k.nr;
  const double dt = k.ctl->dt;
  const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  const bool cell = (j < ns);
  const size_t l = (size_t)i * ns + j;
  if (i == nr) {  // the whole CTA
    if (!cell) return;
    k.vr[l] = 0.0;
    k.vt[l] = 0.0;
    if (k.energy) k.e[l] = 0.0;
    return;
  }
  double vtnew = 0.0;
  if (cell) {
    const size_t lip = l + ns;
    const size_t ljp = (j == ns - 1) ? (size_t)i * ns : l + 1;
    const size_t ljm = (j == 0) ? (size_t)i * ns + ns - 1 : l - 1;
    const size_t lim = (i >= 1) ? l - ns : l;
    // every load first
    const double qr = q_r(k, l, lip);
    const double qt = q_t(k, l, ljp);
    const double qtjm = q_t(k, ljm, l);
    const double qrim = (i >= 1) ? q_r(k, lim, l) : 0.0;
    const double rl = k.rho[l], rlim = k.rho[lim], rjm = k.rho[ljm];
    const double vril = k.vri[l], vtil = k.vti[l];
    const double invdxtheta = k.invdxtheta[i], invdiffrmed = k.invdiffrmed[i];
    double el = 0.0, vrip = 0.0, vtijp = 0.0, invdiffrsup = 0.0;
    if (k.energy) {
      el = k.e[l];
      vrip = k.vri[lip];
      vtijp = k.vti[ljp];
      invdiffrsup = k.invdiffrsup[i];
    }
    if (i >= 1)
      k.vr[l] = vril - dt * 2.0 / (rl + rlim) * (qr - qrim) * invdiffrmed;
    else
      k.vr[l] = 0.0;
    vtnew = vtil - dt * 2.0 / (rl + rjm) * (qt - qtjm) * invdxtheta;
    k.vt[l] = vtnew;
    if (k.energy)
      k.e[l] = el - dt * qr * (vrip - vril) * invdiffrsup - dt * qt * (vtijp - vtil) * invdxtheta;
  }
  if (k.energy && k.beta_cooling) {
    // SubStep3's ring mean of vtheta (SourceEuler.c:1196-1203): this CTA's
    // part, summed in a fixed order
    __shared__ double sh[FB_BS2 / 32];
    double v = cell ? (vtnew + k.rmed[i] * omf(k)) : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
      k.vt_part[(size_t)i * gridDim.x + blockIdx.x] = t;
    }
  }
}

void fb_launch_substep2(const KP &k, cudaStream_t s)
{
  fb_launch(k_substep2, grid2d(k, k.nr + 1), k.cell_bs, 0, s, k);
}

// ------------------------------------------------------------ SubStep3
static __device__ __forceinline__ double vischeat_of(const KP &k, int i, double rho, const Stress &st)
{
  // ComputeViscousHeating, SourceEuler.c:1570-1583 (i >= 1)
  const double viscosity = nu_ring(k, i);
  if (viscosity != 0.0) {
    double vh = 0.5 / viscosity / rho * (st.trr * st.trr + 2.0 * st.trp * st.trp + st.tpp * st.tpp);
    vh += (2.0 / 9.0) * viscosity * rho * st.div * st.div;
    return vh;
  }
  return 0.0;
}

// ComputeViscousTerms on the new velocities (for the heating; DivergenceVelocity
// alone without it), ComputeViscousHeating (SourceEuler.c:1554-1606) and
// SubStep3 (SourceEuler.c:1119-1302; pdV, viscous heating, beta cooling) in
// one pass: a cell's stresses feed its own heating, so they are evaluated
// here (and still stored) instead of read back.  Ring 0's heating is
// extrapolated from rings 1 and 2, whose stresses its threads evaluate too.
// Writes Energy = EnergyNew (ring nr of EnergyNew is never written: zero).
__global__ void __launch_bounds__(FB_BS2) k_substep3(KP k)
{
  fb_grid_dependency();
  const int ns = k.ns, nr = k.nr;
  const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j;
  if (i == nr) {
    k.e[l] = 0.0;
    return;
  }
  const bool heat = k.viscous_heating;
  const Stress st = stress_at(k, k.vr, k.vt, i, j, heat);
  Stress s1, s2;
  double r1 = 0.0, r2 = 0.0;
  if (heat && i == 0) {
    s1 = stress_at(k, k.vr, k.vt, 1, j, true);
    s2 = stress_at(k, k.vr, k.vt, 2, j, true);
    r1 = k.rho[l + ns];
    r2 = k.rho[l + 2 * ns];
  }
  const double el = k.e[l], rl = k.rho[l];
  const double dt = k.ctl->dt;
  double coolfac = 0.0;
  if (k.beta_cooling) {
    // the ring mean of vtheta from SubStep2's partial sums (same CTA width)
    double s = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++) s += k.vt_part[(size_t)i * gridDim.x + b];
    double omega = s;
    omega /= (double)ns;
    omega /= k.rmed[i];
    double coolingtime = k.betatab[i] / omega;
    coolfac = coolingtime;
  }
  k.divv[l] = st.div;
  double vh = 0.0;
  if (heat) {
    k.trr[l] = st.trr;
    k.tpp[l] = st.tpp;
    if (i >= 1) {
      k.trp[l] = st.trp;
      vh = vischeat_of(k, i, rl, st);
    } else {
      // the i = 0 extrapolation tests the viscosity of the last ring visited
      // by the i >= 1 loop (ring nr-1), SourceEuler.c:1598
      const double visc_last = nu_ring(k, nr - 1);
      const double qpip = vischeat_of(k, 1, r1, s1);
      const double qpi2p = vischeat_of(k, 2, r2, s2);
      vh = (visc_last != 0.0) ? qpip * exp(log(qpip / qpi2p) * k.vh_l1 / k.vh_l2) : 0.0;
    }
    k.vischeat[l] = vh;
  }
  const double dv = st.div;
  double en;
  if (k.thermal_cooling) {
    // implicit update with thermal cooling and stellar irradiation
    // (SourceEuler.c:1201-1290); beta cooling does not apply then
    const double tau = 0.5 * k.opacity[l] * rl;
    const double tau_eff = 0.375 * tau + 0.25 * sqrt(3.0) + 0.25 / tau;
    const double temp = (k.gamma - 1.0) * el * (1.0 / rl);
    double num;
    if (k.irradiation) {
      double temp_irr;
      if (k.irradiation == 1) {
        temp_irr = k.irr_ring[i];
      } else {
        // the grazing angle as the reference finally sets it (:1257; the
        // radial temperature gradient computed before it is not used)
        const double albedo = 0.1;
        const double costheta = 0.5 * sqrt(k.rmed[i] * temp) * (2.0 * k.flaringindex);
        const double buf = 0.5 * (tau_eff / k.sigma_sb) * (1.0 - albedo) * k.irr_ring[i] * costheta;
        temp_irr = pow(buf, 0.25);  // NaN stops the step (FB_ERR_NAN); the reference exits
      }
      num = el + dt * (vh * (double)(heat ? 1 : 0) +
                       (2.0 * k.sigma_sb / tau_eff) * (3.0 * pow(temp, 4.0) + pow(temp_irr, 4.0)));
    } else {
      num = el + dt * (vh * (double)(heat ? 1 : 0) + (6.0 * k.sigma_sb / tau_eff) * pow(temp, 4.0));
    }
    const double den = 1.0 + (k.gamma - 1.0) * dt * dv +
                       8.0 * dt * (k.sigma_sb / tau_eff) * (k.gamma - 1.0) * pow(temp, 3.0) * (1.0 / rl);
    en = num / den;
  } else {
    double num = el + (double)(heat ? 1 : 0) * vh * dt;
    double den = 1.0 + (k.gamma - 1.0) * dt * dv;
    en = num / den;
    if (k.temppresc) {  // relaxation towards the initial profile (SourceEuler.c:1162-1175)
      const double coolingtime = k.presc[i];
      num = en + k.energymed[i] * (rl / k.sigmamed[i]) * (dt / coolingtime);
      den = 1.0 + dt / coolingtime;
      en = num / den;
    }
    if (k.beta_cooling) {
      const double d2 = 1.0 + dt / coolfac;  // one per ring: the quotient through its reciprocal
      en = fb_quot(en, d2, 1.0 / d2);
    }
  }
  k.e[l] = en;
}

// ComputeOpacities (SourceEuler.c:1608-1701): Bell & Lin (1994) opacities of
// the cells of rings 0..nr-1 from their temperature and 3-D density, or the
// imposed constant, in code units.
__global__ void __launch_bounds__(FB_BS2) k_opacity(KP k, int constant, double imposed, double factor,
                                                   double unit_temperature, double unit_mass, double inv_l3,
                                                   double conv)
{
  fb_grid_dependency();
  const int ns = k.ns;
  const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j;
  double op;
  if (!constant) {
    const double energ = k.e[l], dens = k.rho[l];
    const double temp = (k.gamma - 1.0) * energ * (1.0 / dens);
    const double phys_temp = temp * unit_temperature;
    const double roversigma = k.rmed[i] / dens;
    const double buf = k.gamma * (k.gamma - 1.0) * energ * pow(roversigma, 3.);
    const double rho3D = 0.5 * pow(buf, -0.5);
    double phys_dens = rho3D * unit_mass * inv_l3;  // kg m^-3 (inv_l3 = pow(unit_length, -3.))
    phys_dens *= 1e-3;                                // g cm^-3
    if (phys_temp < 167.0) {
      op = 2e-4 * pow(phys_temp, 2.0);
    } else if (phys_temp < 203.0) {
      op = 2e16 * pow(phys_temp, -7.0);
    } else if (phys_temp < pow(2e82 * phys_dens, 2. / 49)) {
      op = 0.1 * pow(phys_temp, 0.5);
    } else if (phys_temp < pow(2e89 * pow(phys_dens, 1. / 3), 1. / 27)) {
      op = 2e81 * pow(phys_dens, 1.0) * pow(phys_temp, -24.);
    } else if (phys_temp < pow(1e28 * pow(phys_dens, 1. / 3), 1. / 7)) {
      op = 1e-8 * pow(phys_dens, 2. / 3) * pow(phys_temp, 3.);
    } else if (phys_temp < pow(1.5e56 * pow(phys_dens, 2. / 3), 0.08)) {
      op = 1e-36 * pow(phys_dens, 1. / 3) * pow(phys_temp, 10.);
    } else if (phys_temp < pow(4.31e20 * phys_dens, 2. / 5)) {
      op = 1.5e20 * pow(phys_dens, 1.) * pow(phys_temp, -2.5);
    } else {
      op = 0.348;
    }
    op *= factor;
  } else {
    op = imposed;
  }
  k.opacity[l] = op * conv;
}

void fb_launch_opacity(const KP &k, int constant, double imposed, double factor, double unit_temperature,
                       double unit_mass, double inv_l3, double conv, cudaStream_t s)
{
  fb_launch(k_opacity, grid2d(k, k.nr), k.cell_bs, 0, s, k, constant, imposed, factor, unit_temperature, unit_mass,
            inv_l3, conv);
}

// ComputeOpacities of the current state with the constants held in KP:
// radiative diffusion recomputes the opacity at every substep (in
// ConditionCFL and ComputeRadiativeDiffusion, or in the implicit solver),
// and SubStep3's cooling then uses that one (SourceEuler.c:1326, 1809, 1901)
int fb_launch_opacity_now(const KP &k, cudaStream_t s)
{
  fb_launch(k_opacity, grid2d(k, k.nr), k.cell_bs, 0, s, k, k.op_constant, k.op_imposed, k.op_factor, k.op_utemp,
            k.op_umass, k.op_invl3, k.op_conv);
  return 1;
}

void fb_launch_substep3(const KP &k, cudaStream_t s) { fb_launch(k_substep3, grid2d(k, k.nr + 1), k.cell_bs, 0, s, k); }

// ------------------------------------------------------------ Transport
// Radial pass of the van Leer transport (OneWindRad, TransportEuler.c:124-220
// with ComputeLRMomenta :89-119, ComputeStarRad :141-184, DivisePolarGrid
// SideEuler.c:244-261).  A thread owns one azimuth column and marches
// through a chunk of rings, keeping the slopes and interface values of the
// last rings in registers, so each input is read once and no interface is
// evaluated twice.  Outputs the five (six) transported quantities.
// The quantities of a column are split over two halves of the CTA (warps
// of the first half: RadMomP, RadMomM, ThetaMomP; of the second: ThetaMomM,
// Energy, Rho), so each thread keeps the windows of at most three; both
// halves evaluate the density's own slope and star value.
template <int NQ, int H>
static __device__ __forceinline__ void radial_column(const KP &k, double dt, int j, int i0, int i1)
{
  constexpr int LO = H ? 3 : 0, NH = (H ? NQ : 3) - LO;
  const int ns = k.ns, nr = k.nr;
  const int jp = (j == ns - 1) ? 0 : j + 1;
  const double Om = omf(k);
  const double dtheta = (k.pmax - k.pmin) / (double)ns;
  // window: index 0 = ring k-1, 1 = ring k, 2 = ring k+1
  double W[NH][3], Qo[NH][3], R[3], VW[3];
  double DQ[NH][2], DR[2], QS[NH][2], RS[2], VR[2];
  // flux through the inner face of the cell being updated: the outer-face
  // flux of the cell below, carried from the previous iteration (the face
  // radius Rsup[i-1] is Rinf[i], the same double), so each face's flux is
  // evaluated once
  double FI[NH];
#pragma unroll
  for (int q = 0; q < NH; q++) FI[q] = 0.0;
  // the inputs of one ring, loaded one iteration before they are used,
  // with the ring's table entries: Rmed, InvDiffRmed, Rinf and the
  // InvSurf of the cell below (the one whose update reads this ring's face)
  struct Raw { double r, u0, u1, u2, v, tm, ti, tr, ts; };
  // table windows (slot 1 = ring kk, slot 2 = ring kk+1, TM slot 0 = kk-1)
  double TM[3], TI[3], TR[3], TS[3];
  auto fetch = [&](int kk) -> Raw {
    Raw w = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (kk >= 0 && kk <= nr) {
      w.tm = k.rmed[kk];
      w.ti = k.invdiffrmed[kk];
      w.tr = k.rinf[kk];
      if (kk >= 1) w.ts = k.invsurf[kk - 1];
    }
    if (kk >= 0 && kk <= nr - 1) {
      const size_t l = (size_t)kk * ns + j;
      w.r = k.rho[l];
      if (H == 0) {
        w.u0 = k.vr[l + ns];
        w.u1 = k.vr[l];
        w.u2 = k.vt[(size_t)kk * ns + jp];
      } else {
        w.u0 = k.vt[l];
        if (NQ == 6) w.u1 = k.e[l];
        if (k.vt_copy && kk >= i0 && kk < i1) k.vt_copy[l] = w.u0;  // for the tile variant
      }
    }
    if (kk >= 0 && kk <= nr) w.v = k.vr[(size_t)kk * ns + j];
    return w;
  };
  auto put = [&](const Raw &w, int kk, int slot) {
    VW[slot] = w.v;
    TM[slot] = w.tm;
    TI[slot] = w.ti;
    TR[slot] = w.tr;
    TS[slot] = w.ts;
    if (kk < 0 || kk > nr - 1) {
#pragma unroll
      for (int q = 0; q < NH; q++) { W[q][slot] = 0.0; Qo[q][slot] = 0.0; }
      R[slot] = 0.0;
      return;
    }
    const double r = w.r;
    const double Rm = w.tm;
    double qv[NH];
    if (H == 0) {
      qv[0] = r * w.u0;                    // rp = rho*vr[lip]
      qv[1] = r * w.u1;                    // rm = rho*vr[l]
      qv[2] = r * (w.u2 + Rm * Om) * Rm;   // tp
    } else {
      qv[0] = r * (w.u0 + Rm * Om) * Rm;   // tm
      if (NQ == 6) qv[1] = w.u1;
      qv[NH - 1] = r;
    }
    const double den = r + 1e-20, rden = fb_rcp(den);
#pragma unroll
    for (int q = 0; q < NH; q++) { Qo[q][slot] = qv[q]; W[q][slot] = fb_quot(qv[q], den, rden); }  // qv / den
    R[slot] = r;
  };
  auto slope = [&](double am, double a0, double ap, int kk) -> double {
    if (kk <= 0 || kk >= nr - 1) return 0.0;
    double dqm = (a0 - am) * TI[1];  // InvDiffRmed[kk]
    double dqp = (ap - a0) * TI[2];  // InvDiffRmed[kk + 1]
    if (dqp * dqm > 0.0) return fb_vl_quot(2.0 * dqp * dqm, dqp + dqm);
    return 0.0;
  };
  int kstart = max(i0 - 1, 0);
  Raw nxt = fetch(kstart + 1);
  put(fetch(kstart - 1), kstart - 1, 0);
  put(fetch(kstart), kstart, 1);
#pragma unroll
  for (int q = 0; q < NH; q++) { DQ[q][0] = 0.0; QS[q][0] = 0.0; }
  DR[0] = 0.0; RS[0] = 0.0; VR[0] = 0.0;
  for (int kk = kstart; kk <= i1; kk++) {
    const Raw cur = nxt;
    nxt = fetch(kk + 2);
    put(cur, kk + 1, 2);
    const double vrk = VW[1];  // vr of ring kk
    const double rmk = TM[1];
    const double rmkm = TM[0];  // 0 below ring 0
#pragma unroll
    for (int q = 0; q < NH; q++) DQ[q][1] = slope(W[q][0], W[q][1], W[q][2], kk);
    DR[1] = slope(R[0], R[1], R[2], kk);
    if (kk == 0 || kk >= nr) {
#pragma unroll
      for (int q = 0; q < NH; q++) QS[q][1] = 0.0;
      RS[1] = 0.0;
    } else if (vrk > 0.0) {
      const double f = (rmk - rmkm - vrk * dt) * 0.5;
#pragma unroll
      for (int q = 0; q < NH; q++) QS[q][1] = W[q][0] + (rmk - rmkm - vrk * dt) * 0.5 * DQ[q][0];
      RS[1] = R[0] + f * DR[0];
    } else {
      const double rmkp = TM[2];
      const double f = (rmkp - rmk + vrk * dt) * 0.5;
#pragma unroll
      for (int q = 0; q < NH; q++) QS[q][1] = W[q][1] - (rmkp - rmk + vrk * dt) * 0.5 * DQ[q][1];
      RS[1] = R[1] - f * DR[1];
    }
    VR[1] = vrk;
    const int io = kk - 1;
    // VanLeerRadial (TransportEuler.c:205-212): varq = dt dtheta Rinf[i]
    // QStar RhoStar Vrad at face i minus the same at face i+1
    const double b = dt * dtheta * TR[1];  // Rinf[kk]: face kk = outer face of cell io
    double FO[NH];
#pragma unroll
    for (int q = 0; q < NH; q++) FO[q] = b * QS[q][1] * RS[1] * VR[1];
    if (io >= i0 && io < i1) {
      const size_t l = (size_t)io * ns + j;
#pragma unroll
      for (int q = 0; q < NH; q++) {
        double varq = FI[q];
        varq -= FO[q];
        k.q[LO + q][l] = Qo[q][0] + varq * TS[1];  // InvSurf[io]
        if (LO + q == NQ - 1 && io == 0) k.lost0[j] = varq;
      }
    }
#pragma unroll
    for (int q = 0; q < NH; q++) FI[q] = FO[q];
    // shift windows
#pragma unroll
    for (int q = 0; q < NH; q++) {
      W[q][0] = W[q][1]; W[q][1] = W[q][2];
      Qo[q][0] = Qo[q][1]; Qo[q][1] = Qo[q][2];
      DQ[q][0] = DQ[q][1];
      QS[q][0] = QS[q][1];
    }
    R[0] = R[1]; R[1] = R[2];
    VW[0] = VW[1]; VW[1] = VW[2];
    TM[0] = TM[1]; TM[1] = TM[2];
    TI[1] = TI[2];
    TR[1] = TR[2];
    TS[1] = TS[2];
    DR[0] = DR[1];
    RS[0] = RS[1];
    VR[0] = VR[1];
  }
}

// CTAs of 2 tx threads: columns blockIdx.x tx .. + tx, rings of one chunk
template <int NQ>
__global__ void __launch_bounds__(256, 2) k_transport_radial(KP k, double dtov, int chunk)
{
  fb_grid_dependency();
  const double dt = dt_of(k, dtov);
  const int tx = blockDim.x >> 1, h = (threadIdx.x >= tx) ? 1 : 0;  // tx % 32 == 0: warp-uniform
  const int j = blockIdx.x * tx + threadIdx.x - h * tx;
  if (j >= k.ns) return;
  const int i0 = blockIdx.y * chunk;
  const int i1 = min(k.nr, i0 + chunk);
  if (h == 0)
    radial_column<NQ, 0>(k, dt, j, i0, i1);
  else
    radial_column<NQ, 1>(k, dt, j, i0, i1);
}

// Sum over the block for any blockDim that is a multiple of 32.
static __device__ double block_sum_dyn(double v, double *sh)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (lane < nw) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[0] = v;
  }
  __syncthreads();
  double r = sh[0];
  __syncthreads();
  return r;
}


// Azimuthal pass (OneWindTheta, TransportEuler.c:226-247): ring mean,
// residual and integer FARGO shift (:249-373), van Leer on the residual and
// on the uniform part (:375-465), the shift itself, then ComputeVelocities'
// vtheta (:515-547), the energy floor (SourceEuler.c:2524) and the
// sub-Keplerian edge rings (SideEuler.c:1008-1044).
//
// One CTA per ring with the ring's NQ quantities in shared memory.  Thread t
// owns the E cells t, t+T, t+2T, ... (T = blockDim.x), so every shared-memory
// sweep is bank-conflict free and a ring of up to 1024*E cells keeps 24-32
// warps busy.  Per pass and quantity the face values go through two
// shared-memory stages: W = q/(RhoInt+1e-20) for the own cells, then the van
// Leer slope DQ of the own cells; each thread then forms the upwind values at
// both faces of its cells and updates them (three barriers per quantity).
// The density slopes of RhoStar share the DQ ring.  The arithmetic is the
// reference's, term for term (ComputeStarTheta :392-433, VanLeerTheta
// :435-465); only the work split differs.
//
// shared memory: NQ rings of quantities, the residual velocity, W, DQ --
// 110.6 KB for six quantities of 1536 cells, so that two CTAs share an SM
//
// The wide variant (where 2 NQ + 1 rings fit) goes through the quantities
// together: W of every quantity in place of the quantity's ring (its value
// kept in registers), one slope ring per quantity, the updates held in
// registers until every read of W is done -- five barriers per pass instead
// of three per quantity, and NQ independent chains in every phase.
#define FB_AZI_RINGS(NQ) ((NQ) + 3)
#define FB_AZI_RINGS_WIDE(NQ) (2 * (NQ) + 1)
template <int E, bool WIDE> struct AziMaxThreads { static const int value = (E == 1 || (E == 2 && !WIDE)) ? 1024 : 768; };
template <int NQ, int E, bool FULL, bool WIDE>
__global__ void __launch_bounds__(AziMaxThreads<E, WIDE>::value) k_transport_azimuthal(KP k, double dtov)
{
  fb_grid_dependency();
  extern __shared__ double smem[];
  __shared__ double sh[32];
  const double dt = dt_of(k, dtov);
  const int i = blockIdx.x, ns = k.ns, nr = k.nr, T = blockDim.x, tid = threadIdx.x;
  const size_t base = (size_t)i * ns;
  double *Q = smem;              // NQ rings
  double *vres = Q + NQ * ns;    // residual azimuthal velocity
  double *W = vres + ns;         // q / RhoInt (narrow variant)
  double *D = vres + (WIDE ? 1 : 2) * ns;  // van Leer slopes of W (wide: NQ rings)
  double *DR = D;                // density slopes (RhoStar), read before D is rewritten
  for (int j = tid; j < ns; j += T)
    for (int q = 0; q < NQ; q++) Q[q * ns + j] = k.q[q][base + j];
  // ComputeThetaElongations / ComputeAverageThetaVelocities / ComputeResiduals
  const double invdt = 1.0 / dt;
  double s = 0.0;
  for (int j = tid; j < ns; j += T) {
    double elong = k.vt[base + j] * dt;
    s += elong * invdt;
  }
  s = block_sum_dyn(s, sh);
  const double VMed = s / (double)ns;
  // ComputeConstantResidual (TransportEuler.c:310-348)
  const double dpinvns = (k.pmax - k.pmin) / (double)ns;
  const double Ntilde = VMed * k.invrmed[i] * dt * (double)ns / (k.pmax - k.pmin);
  const double Nround = floor(Ntilde + 0.5);
  const long nshift = (long)Nround;
  double vconst = (Ntilde - Nround) * k.rmed[i] * invdt * dpinvns;
  for (int j = tid; j < ns; j += T) {
    double elong = k.vt[base + j] * dt;
    double v = elong * invdt - VMed;
    if (!k.fast_transport) v = vconst + v;
    vres[j] = v;
  }
  if (!k.fast_transport) vconst = 0.0;
  const double dxtheta = k.dxtheta[i], invdxtheta = k.invdxtheta[i];
  const double dxrad = (k.rsup[i] - k.rinf[i]) * dt;
  const double invsurf = 1.0 / k.surf[i];
  const double *rho = Q + (NQ - 1) * ns;
  // own cells j = tid + e T (all valid when FULL: ns == E T) and their
  // periodic neighbours
  int jj[E], jjm[E], jjp[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int j = tid + e * T;
    jj[e] = j;
    jjm[e] = (j == 0) ? ns - 1 : j - 1;
    jjp[e] = (j == ns - 1) ? 0 : j + 1;
  }
#define OWN(e) (FULL || jj[e] < ns)
  for (int pass = 0; pass < 2; pass++) {
    const bool uniform = (pass == 1);
    if (uniform && !k.fast_transport) break;  // NoSplitAdvection: no update
    __syncthreads();  // Q and vres complete
    // RhoStar (ComputeStarTheta(Rho, V, RhoStar)); RhoInt is the density
    // before this pass, kept in registers for the own cells.
    double R[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      const double rm = rho[jjm[e]], r0 = rho[jj[e]], rp = rho[jjp[e]];
      R[e] = r0;
      const double dqm = (r0 - rm), dqp = (rp - r0);
      DR[jj[e]] = (dqp * dqm > 0.0) ? fb_vl_quot(dqp * dqm, dqp + dqm) * invdxtheta : 0.0;
    }
    __syncthreads();
    // Per face, the upwind cell u and the factor f of its star value:
    // (kl > 0) ? q[j-1] + (dxtheta - kl) DQ[j-1] : q[j] - (dxtheta + kl) DQ[j]
    // is q[u] + f DQ[u] with f = dxtheta - kl or -(dxtheta + kl) (the same
    // value: negation and a + (-b) = a - b are exact).
    double RSl[E], RSh[E], Vl[E], Vh[E], fl[E], fh[E], den[E], rden[E];
    int ul[E], uh[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      const double vl = uniform ? vconst : vres[jj[e]], vh = uniform ? vconst : vres[jjp[e]];
      Vl[e] = vl;
      Vh[e] = vh;
      const double kl = vl * dt, kh = vh * dt;
      ul[e] = (kl > 0.0) ? jjm[e] : jj[e];
      fl[e] = (kl > 0.0) ? (dxtheta - kl) : -(dxtheta + kl);
      uh[e] = (kh > 0.0) ? jj[e] : jjp[e];
      fh[e] = (kh > 0.0) ? (dxtheta - kh) : -(dxtheta + kh);
      RSl[e] = rho[ul[e]] + fl[e] * DR[ul[e]];
      RSh[e] = rho[uh[e]] + fh[e] * DR[uh[e]];
      den[e] = R[e] + 1e-20;
      rden[e] = 1.0 / den[e];
    }
    if constexpr (WIDE) {
      double q0[NQ][E];
      __syncthreads();  // every read of rho and DR done: W replaces the rings, DR is D[0]
#pragma unroll
      for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int e = 0; e < E; e++) {
          if (!OWN(e)) continue;
          double *qb = Q + q * ns;
          q0[q][e] = qb[jj[e]];
          qb[jj[e]] = fb_quot(q0[q][e], den[e], rden[e]);  // W = q0 / (RhoInt + 1e-20)
        }
      __syncthreads();  // W complete
#pragma unroll
      for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int e = 0; e < E; e++) {
          if (!OWN(e)) continue;
          const double *Wq = Q + q * ns;
          const double w0 = Wq[jj[e]];
          const double dqm = (w0 - Wq[jjm[e]]), dqp = (Wq[jjp[e]] - w0);
          D[q * ns + jj[e]] = (dqp * dqm > 0.0) ? fb_vl_quot(dqp * dqm, dqp + dqm) * invdxtheta : 0.0;
        }
      __syncthreads();  // DQ complete
#pragma unroll
      for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int e = 0; e < E; e++) {
          if (!OWN(e)) continue;
          const double *Wq = Q + q * ns, *Dq = D + q * ns;
          const double qsl = Wq[ul[e]] + fl[e] * Dq[ul[e]];
          const double qsh = Wq[uh[e]] + fh[e] * Dq[uh[e]];
          double varq = dxrad * qsl * RSl[e] * Vl[e];
          varq -= dxrad * qsh * RSh[e] * Vh[e];
          q0[q][e] = q0[q][e] + varq * invsurf;
        }
      __syncthreads();  // every read of W done
#pragma unroll
      for (int q = 0; q < NQ; q++)
#pragma unroll
        for (int e = 0; e < E; e++)
          if (OWN(e)) Q[q * ns + jj[e]] = q0[q][e];
    } else {
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      double *qb = Q + q * ns;
      double q0[E];
      if (q > 0) __syncthreads();  // every read of the previous W and DQ done
#pragma unroll
      for (int e = 0; e < E; e++) {
        if (!OWN(e)) continue;
        q0[e] = qb[jj[e]];
        W[jj[e]] = fb_quot(q0[e], den[e], rden[e]);  // q0 / (RhoInt + 1e-20)
      }
      __syncthreads();  // W complete (and, for q = 0, every read of DR done)
#pragma unroll
      for (int e = 0; e < E; e++) {
        if (!OWN(e)) continue;
        const double w0 = W[jj[e]];
        const double dqm = (w0 - W[jjm[e]]), dqp = (W[jjp[e]] - w0);
        D[jj[e]] = (dqp * dqm > 0.0) ? fb_vl_quot(dqp * dqm, dqp + dqm) * invdxtheta : 0.0;
      }
      __syncthreads();  // DQ complete
#pragma unroll
      for (int e = 0; e < E; e++) {
        if (!OWN(e)) continue;
        const double qsl = W[ul[e]] + fl[e] * D[ul[e]];
        const double qsh = W[uh[e]] + fh[e] * D[uh[e]];
        double varq = dxrad * qsl * RSl[e] * Vl[e];
        varq -= dxrad * qsh * RSh[e] * Vh[e];
        qb[jj[e]] = q0[e] + varq * invsurf;
      }
    }
    }
  }
#undef OWN
#define jc(e) (tid + (e) * T)  // own cells (valid while < ns)
  __syncthreads();
  // AdvectSHIFT (TransportEuler.c:350-373) for every quantity: cell j takes
  // cell (j - nshift) mod ns
  int shift = (int)(nshift % ns);
  if (shift < 0) shift += ns;
  for (int q = 0; q < NQ; q++) {
    double *qb = Q + q * ns;
    double tmp[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int j = jc(e);
      int ji = j - shift;
      if (ji < 0) ji += ns;
      tmp[e] = (j < ns) ? qb[ji] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; e++)
      if (jc(e) < ns) qb[jc(e)] = tmp[e];
  }
  __syncthreads();
  // ComputeVelocities, vtheta part; floors on energy; sub-Keplerian edges
  const double *tp = Q + 2 * ns, *tm = Q + 3 * ns;
  const int subkep = (!k.transport_only) && (i == 0 || i == nr - 1);
  for (int j = tid; j < ns; j += T) {
    const int jm = (j == 0) ? ns - 1 : j - 1;
    double v = (tp[jm] + tm[j]) / (rho[j] + rho[jm] + 1e-20) / k.rmed[i] - k.rmed[i] * omf(k);
    if (subkep) v = k.vthetamed[i] - k.rmed[i] * omf(k);
    k.vt[base + j] = v;
    k.rho_t[base + j] = rho[j];
    k.q[0][base + j] = Q[j];
    k.q[1][base + j] = Q[ns + j];
    if (NQ == 6) {
      double e = Q[4 * ns + j];
      if (k.add_floors && !k.transport_only) {
        double e_bottom = 1e-3 * k.energymed[i];
        if (e < e_bottom) e = e_bottom;
      }
      k.e[base + j] = e;
    }
  }
#undef jc
}

// Packed variant of the azimuthal pass: the same phases as the wide variant,
// with cell j's quantities side by side at P[6j .. 6j+5] (RadMomP, RadMomM,
// ThetaMomP, ThetaMomM, [Energy,] Rho; without energy the sixth slot is
// unused) and their slopes likewise, so one address per face serves every
// quantity through 16-byte shared accesses, two quantities at a time
// (48-byte cells: conflict-free per quarter warp).  The residual velocity
// is recomputed from vtheta where it is needed, and without energy the
// density slopes of RhoStar live in the unused sixth slot, so the variant
// takes 2 x 6 (+ 1 with energy) rings of nsec doubles: 221 KB for 2304
// isothermal cells.
#define AZP 6
#define AZP_RINGS(NQ) (2 * AZP + ((NQ) == 6 ? 1 : 0))
template <int NQ, int E, bool FULL>
__global__ void __launch_bounds__((E == 1) ? 1024 : 768) k_transport_azimuthal_packed(KP k, double dtov)
{
  fb_grid_dependency();
  extern __shared__ double2 smem2[];
  __shared__ double sh[32];
  const double dt = dt_of(k, dtov);
  const int i = blockIdx.x, ns = k.ns, nr = k.nr, T = blockDim.x, tid = threadIdx.x;
  const size_t base = (size_t)i * ns;
  constexpr int RH = NQ - 1;          // slot of the density
  double *P = (double *)smem2;        // ns cells x 6
  double *PD = P + AZP * ns;          // slopes, ns x 6
  // density slopes (RhoStar): slot 5 of the cells without energy, a ring of
  // their own with it
  double *DRb = (NQ == 6) ? PD + AZP * ns : P + 5;
  const int drs = (NQ == 6) ? 1 : AZP;
#define DR_AT(j) DRb[(size_t)(j) * drs]
  // a cell's slot pair (2h, 2h+1) as one 16-byte access: 48-byte cells keep
  // these free of bank conflicts, single 8-byte slots would not be
  auto pair = [&](const double *A, int j, int h) -> double2 { return ((const double2 *)(A + AZP * j))[h]; };
  auto rho_at = [&](int j) -> double {
    const double2 x = pair(P, j, RH / 2);
    return (RH & 1) ? x.y : x.x;
  };
  int jj[E], jjm[E], jjp[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int j = tid + e * T;
    jj[e] = j;
    jjm[e] = (j == 0) ? ns - 1 : j - 1;
    jjp[e] = (j == ns - 1) ? 0 : j + 1;
  }
#define OWN(e) (FULL || jj[e] < ns)
  // every global load of the kernel at once: the own cells' quantities and
  // vtheta of each own cell and of its upper neighbour (the residual
  // velocities of both faces)
  double vtc[E], vtn[E];
  {
    double v[E][AZP];
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
#pragma unroll
      for (int q = 0; q < AZP; q++) v[e][q] = (q < NQ) ? k.q[q][base + jj[e]] : 0.0;
      vtc[e] = k.vt[base + jj[e]];
      vtn[e] = k.vt[base + jjp[e]];
    }
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      double2 *c = (double2 *)(P + AZP * jj[e]);
#pragma unroll
      for (int h = 0; h < AZP / 2; h++) c[h] = make_double2(v[e][2 * h], v[e][2 * h + 1]);
    }
  }
  // ComputeThetaElongations / ComputeAverageThetaVelocities / ComputeResiduals
  const double invdt = 1.0 / dt;
  double s = 0.0;
#pragma unroll
  for (int e = 0; e < E; e++) {
    if (!OWN(e)) continue;
    double elong = vtc[e] * dt;
    s += elong * invdt;
  }
  s = block_sum_dyn(s, sh);
  const double VMed = s / (double)ns;
  // ComputeConstantResidual (TransportEuler.c:310-348)
  const double dpinvns = (k.pmax - k.pmin) / (double)ns;
  const double Ntilde = VMed * k.invrmed[i] * dt * (double)ns / (k.pmax - k.pmin);
  const double Nround = floor(Ntilde + 0.5);
  const long nshift = (long)Nround;
  double vconst = (Ntilde - Nround) * k.rmed[i] * invdt * dpinvns;
  const double vconst0 = vconst;
  // ComputeResiduals' value of a cell of vtheta vtj
  auto vres_of = [&](double vtj) -> double {
    double elong = vtj * dt;
    double v = elong * invdt - VMed;
    if (!k.fast_transport) v = vconst0 + v;
    return v;
  };
  if (!k.fast_transport) vconst = 0.0;
  const double dxtheta = k.dxtheta[i], invdxtheta = k.invdxtheta[i];
  const double dxrad = (k.rsup[i] - k.rinf[i]) * dt;
  const double invsurf = 1.0 / k.surf[i];
  for (int pass = 0; pass < 2; pass++) {
    const bool uniform = (pass == 1);
    if (uniform && !k.fast_transport) break;  // NoSplitAdvection: no update
    __syncthreads();  // P complete
    // RhoStar (ComputeStarTheta(Rho, V, RhoStar)); RhoInt in registers
    double R[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      // single-slot reads: slot 5 of a neighbour may be getting its slope
      const double rm = P[AZP * jjm[e] + RH], r0 = P[AZP * jj[e] + RH], rp = P[AZP * jjp[e] + RH];
      R[e] = r0;
      const double dqm = (r0 - rm), dqp = (rp - r0);
      DR_AT(jj[e]) = (dqp * dqm > 0.0) ? fb_vl_quot(dqp * dqm, dqp + dqm) * invdxtheta : 0.0;
    }
    __syncthreads();
    // per face the upwind cell u and the factor f of its star value (as in
    // the other variants)
    double RSl[E], RSh[E], Vl[E], Vh[E], fl[E], fh[E], den[E], rden[E];
    int ul[E], uh[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      const double vl = uniform ? vconst : vres_of(vtc[e]), vh = uniform ? vconst : vres_of(vtn[e]);
      Vl[e] = vl;
      Vh[e] = vh;
      const double kl = vl * dt, kh = vh * dt;
      ul[e] = (kl > 0.0) ? jjm[e] : jj[e];
      fl[e] = (kl > 0.0) ? (dxtheta - kl) : -(dxtheta + kl);
      uh[e] = (kh > 0.0) ? jj[e] : jjp[e];
      fh[e] = (kh > 0.0) ? (dxtheta - kh) : -(dxtheta + kh);
      RSl[e] = rho_at(ul[e]) + fl[e] * DR_AT(ul[e]);
      RSh[e] = rho_at(uh[e]) + fh[e] * DR_AT(uh[e]);
      den[e] = R[e] + 1e-20;
      rden[e] = 1.0 / den[e];
    }
    double q0[E][AZP];
    __syncthreads();  // every read of rho and DR done: W replaces the cells (and slot 5)
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      double2 *c = (double2 *)(P + AZP * jj[e]);
#pragma unroll
      for (int h = 0; h < AZP / 2; h++) {
        const double2 x = c[h];
        q0[e][2 * h] = x.x;
        q0[e][2 * h + 1] = x.y;
        const double wa = (2 * h < NQ) ? fb_quot(x.x, den[e], rden[e]) : 0.0;  // q0 / den
        const double wb = (2 * h + 1 < NQ) ? fb_quot(x.y, den[e], rden[e]) : 0.0;
        c[h] = make_double2(wa, wb);
      }
    }
    __syncthreads();  // W complete
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      const double2 *cm = (const double2 *)(P + AZP * jjm[e]), *c0 = (const double2 *)(P + AZP * jj[e]),
                    *cp = (const double2 *)(P + AZP * jjp[e]);
      double2 *dd = (double2 *)(PD + AZP * jj[e]);
#pragma unroll
      for (int h = 0; h < AZP / 2; h++) {
        const double2 wm = cm[h], w0 = c0[h], wp = cp[h];
        const double m_[2] = {wm.x, wm.y}, z_[2] = {w0.x, w0.y}, p_[2] = {wp.x, wp.y};
        double d2[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const double dqm = (z_[u] - m_[u]), dqp = (p_[u] - z_[u]);
          d2[u] = (2 * h + u < NQ && dqp * dqm > 0.0) ? fb_vl_quot(dqp * dqm, dqp + dqm) * invdxtheta : 0.0;
        }
        dd[h] = make_double2(d2[0], d2[1]);
      }
    }
    __syncthreads();  // DQ complete
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      const double2 *cwl = (const double2 *)(P + AZP * ul[e]), *cdl = (const double2 *)(PD + AZP * ul[e]);
      const double2 *cwh = (const double2 *)(P + AZP * uh[e]), *cdh = (const double2 *)(PD + AZP * uh[e]);
#pragma unroll
      for (int h = 0; h < AZP / 2; h++) {
        const double2 wl = cwl[h], dl = cdl[h], wh = cwh[h], dh = cdh[h];
        const double wl_[2] = {wl.x, wl.y}, dl_[2] = {dl.x, dl.y}, wh_[2] = {wh.x, wh.y}, dh_[2] = {dh.x, dh.y};
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int q = 2 * h + u;
          if (q >= NQ) continue;
          const double qsl = wl_[u] + fl[e] * dl_[u];
          const double qsh = wh_[u] + fh[e] * dh_[u];
          double varq = dxrad * qsl * RSl[e] * Vl[e];
          varq -= dxrad * qsh * RSh[e] * Vh[e];
          q0[e][q] = q0[e][q] + varq * invsurf;
        }
      }
    }
    __syncthreads();  // every read of W done
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      double2 *c = (double2 *)(P + AZP * jj[e]);
#pragma unroll
      for (int h = 0; h < AZP / 2; h++) c[h] = make_double2(q0[e][2 * h], q0[e][2 * h + 1]);
    }
  }
  __syncthreads();
  // AdvectSHIFT (TransportEuler.c:350-373): cell j takes cell (j - nshift) mod ns
  int shift = (int)(nshift % ns);
  if (shift < 0) shift += ns;
  {
    double2 tmp[E][AZP / 2];
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      int ji = jj[e] - shift;
      if (ji < 0) ji += ns;
      const double2 *c = (const double2 *)(P + AZP * ji);
#pragma unroll
      for (int h = 0; h < AZP / 2; h++) tmp[e][h] = c[h];
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (!OWN(e)) continue;
      double2 *c = (double2 *)(P + AZP * jj[e]);
#pragma unroll
      for (int h = 0; h < AZP / 2; h++) c[h] = tmp[e][h];
    }
  }
#undef OWN
#undef DR_AT
  __syncthreads();
  // ComputeVelocities, vtheta part; floors on energy; sub-Keplerian edges
  const int subkep = (!k.transport_only) && (i == 0 || i == nr - 1);
  for (int j = tid; j < ns; j += T) {
    const int jm = (j == 0) ? ns - 1 : j - 1;
    const double2 c0 = pair(P, j, 0), c1 = pair(P, j, 1), c2 = pair(P, j, 2), m1 = pair(P, jm, 1), m2 = pair(P, jm, 2);
    const double rj = (RH & 1) ? c2.y : c2.x, rjm = (RH & 1) ? m2.y : m2.x;  // RH is 4 or 5
    double v = (m1.x + c1.y) / (rj + rjm + 1e-20) / k.rmed[i] - k.rmed[i] * omf(k);  // tp[jm] + tm[j]
    if (subkep) v = k.vthetamed[i] - k.rmed[i] * omf(k);
    k.vt[base + j] = v;
    k.rho_t[base + j] = rj;
    k.q[0][base + j] = c0.x;
    k.q[1][base + j] = c0.y;
    if (NQ == 6) {
      double e = c2.x;
      if (k.add_floors && !k.transport_only) {
        double e_bottom = 1e-3 * k.energymed[i];
        if (e < e_bottom) e = e_bottom;
      }
      k.e[base + j] = e;
    }
  }
}

// Register variant of the azimuthal pass (variant 4).  Thread t owns the E
// contiguous cells c0 = t E .. t E + E - 1 of its ring (nsec = E T with T a
// multiple of 32); every quantity of its cells stays in registers, loaded as
// 16-byte pairs along the azimuth.  A neighbour's value crosses lanes by a
// warp shuffle and warps through a small double-buffered halo in shared
// memory (one barrier per exchange).  Each face flux is evaluated once, by the
// owner of the cell above the face, and reaches the cell below through the
// next exchange; the quantities are advanced one after another, so only one
// quantity's quotients, slopes and fluxes are live at a time.  The arithmetic
// is that of the other variants, operation for operation, and the ring mean
// adds the same cells in the same order (thread t's cells t, t + T, ...), so
// for the same E the results agree to the last bit.
#define AZR_MAXW 32  // warps per CTA
#define AZR_NV 2     // values per exchange and side
#define AZR_MAXT 768  // threads per CTA (each kernel instance is bounded by its own MT <= 768)

// The left neighbour's last-cell values rL (nl of them, from sL of the thread
// before) and the right neighbour's first-cell values rR (from sR of the
// thread after), around the ring.
template <int NL, int NR>
static __device__ __forceinline__ void azr_exchange(double (*hal)[2][AZR_MAXW][AZR_NV], int &xb, int lane, int w,
                                                    int wl, int wr, const double *sL, double *rL, const double *sR,
                                                    double *rR)
{
#pragma unroll
  for (int v = 0; v < NL; v++) rL[v] = __shfl_up_sync(0xffffffffu, sL[v], 1);
#pragma unroll
  for (int v = 0; v < NR; v++) rR[v] = __shfl_down_sync(0xffffffffu, sR[v], 1);
  if (lane == 31)
#pragma unroll
    for (int v = 0; v < NL; v++) hal[xb][0][w][v] = sL[v];
  if (lane == 0)
#pragma unroll
    for (int v = 0; v < NR; v++) hal[xb][1][w][v] = sR[v];
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int v = 0; v < NL; v++) rL[v] = hal[xb][0][wl][v];
  if (lane == 31)
#pragma unroll
    for (int v = 0; v < NR; v++) rR[v] = hal[xb][1][wr][v];
  xb ^= 1;
}

template <int E>
static __device__ __forceinline__ void azr_load(const double *p, double (&v)[E])
{
  if ((E & 1) == 0) {
#pragma unroll
    for (int h = 0; h < E / 2; h++) {
      const double2 x = ((const double2 *)p)[h];
      v[2 * h] = x.x;
      v[2 * h + 1] = x.y;
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = p[e];
  }
}

// One ring of the register variant: the quantities q0 and vtheta vt of the
// thread's own cells (loaded by the caller), vs = vtheta of cells tid, tid + T,
// ... (the ring mean's order).  The results of own cell c0 + e land at cell
// p = c0 + e + nshift (mod nsec): out(e, p, vtheta, density, RadMomP,
// RadMomM, energy).
// The ring's entries of the 1-D tables, loaded together with the ring's
// fields (not one by one where the arithmetic first needs them).
struct AzrTab {
  double invrmed, rmed, dxtheta, invdxtheta, rsup, rinf, surf, vthetamed, energymed;
};
static __device__ __forceinline__ AzrTab azr_tab(const KP &k, int i)
{
  AzrTab t;
  t.invrmed = k.invrmed[i];
  t.rmed = k.rmed[i];
  t.dxtheta = k.dxtheta[i];
  t.invdxtheta = k.invdxtheta[i];
  t.rsup = k.rsup[i];
  t.rinf = k.rinf[i];
  t.surf = k.surf[i];
  t.vthetamed = k.vthetamed ? k.vthetamed[i] : 0.0;
  t.energymed = (k.energy && k.energymed) ? k.energymed[i] : 0.0;
  return t;
}

// Neighbour values within one warp only (the tile variant): lane 0's left
// and lane 31's right neighbours are its own values, which only the tile's
// halo cells read.
template <int NL, int NR>
static __device__ __forceinline__ void azt_exchange(const double *sL, double *rL, const double *sR, double *rR)
{
#pragma unroll
  for (int v = 0; v < NL; v++) rL[v] = __shfl_up_sync(0xffffffffu, sL[v], 1);
#pragma unroll
  for (int v = 0; v < NR; v++) rR[v] = __shfl_down_sync(0xffffffffu, sR[v], 1);
}

// TILE = false: the register variant, one CTA per ring, c0 = tid E, the ring
// mean from vs by one CTA reduction, neighbours across warps through hal.
// TILE = true: the tile variant, one warp per tile of the ring, c0 = the
// ring cell of the warp's first loaded cell plus lane E (any integer: taken
// modulo nsec), the ring mean vmed_in given, no barrier at all.
template <int NQ, int E, bool TILE, class Out>
static __device__ __forceinline__ void azr_ring(const KP &k, double dt, int i, const AzrTab &tb,
                                                double (&q0)[NQ][E], const double (&vt)[E], const double (&vs)[E],
                                                double vmed_in, int c0, double *sh,
                                                double (*hal)[2][AZR_MAXW][AZR_NV], int &xb, Out out)
{
  const int ns = k.ns, nr = k.nr, T = blockDim.x, tid = threadIdx.x;
  const int lane = tid & 31, w = tid >> 5, nw = T >> 5;
  const int wl = (w == 0) ? nw - 1 : w - 1, wr = (w == nw - 1) ? 0 : w + 1;
  constexpr int RH = NQ - 1;  // the density is the last quantity
#define AZR_X(NL, NR, sL, rL, sR, rR)                                       \
  do {                                                                      \
    if (TILE)                                                               \
      azt_exchange<NL, NR>(sL, rL, sR, rR);                                 \
    else                                                                    \
      azr_exchange<NL, NR>(hal, xb, lane, w, wl, wr, sL, rL, sR, rR);       \
  } while (0)
  // ComputeThetaElongations / ComputeAverageThetaVelocities / ComputeResiduals
  const double invdt = 1.0 / dt;
  double VMed = vmed_in;
  if (!TILE) {
    double s = 0.0;
#pragma unroll
    for (int e = 0; e < E; e++) {
      double elong = vs[e] * dt;
      s += elong * invdt;
    }
    s = block_sum_dyn(s, sh);
    VMed = s / (double)ns;
  }
  // ComputeConstantResidual (TransportEuler.c:310-348)
  const double dpinvns = (k.pmax - k.pmin) / (double)ns;
  const double Ntilde = VMed * tb.invrmed * dt * (double)ns / (k.pmax - k.pmin);
  const double Nround = floor(Ntilde + 0.5);
  const long nshift = (long)Nround;
  double vconst = (Ntilde - Nround) * tb.rmed * invdt * dpinvns;
  const double vconst0 = vconst;
  auto vres_of = [&](double vtj) -> double {
    double elong = vtj * dt;
    double v = elong * invdt - VMed;
    if (!k.fast_transport) v = vconst0 + v;
    return v;
  };
  if (!k.fast_transport) vconst = 0.0;
  const double dxtheta = tb.dxtheta, invdxtheta = tb.invdxtheta;
  const double dxrad = (tb.rsup - tb.rinf) * dt;
  const double invsurf = 1.0 / tb.surf;
  for (int pass = 0; pass < 2; pass++) {
    const bool uniform = (pass == 1);
    if (uniform && !k.fast_transport) break;  // NoSplitAdvection: no update
    // lower face e of the own cell c0 + e: velocity, upwind side (left when
    // the displacement is positive) and the factor of its star value
    double V[E], f[E];
    bool upl[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      V[e] = uniform ? vconst : vres_of(vt[e]);
      const double kf = V[e] * dt;
      upl[e] = (kf > 0.0);
      f[e] = upl[e] ? (dxtheta - kf) : -(dxtheta + kf);
    }
    // RhoStar (ComputeStarTheta(Rho, V, RhoStar)): density slopes
    double rL[1], rR[1];
    {
      const double sL[1] = {q0[RH][E - 1]}, sR[1] = {q0[RH][0]};
      AZR_X(1, 1, sL, rL, sR, rR);
    }
    double DR[E], den[E], rden[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const double rm = (e == 0) ? rL[0] : q0[RH][e - 1], r0 = q0[RH][e];
      const double rp = (e == E - 1) ? rR[0] : q0[RH][e + 1];
      const double dqm = (r0 - rm), dqp = (rp - r0);
      DR[e] = fb_vl_slope(dqm, dqp, invdxtheta);
      den[e] = r0 + 1e-20;
      rden[e] = fb_rcp(den[e]);
    }
    // quotients q / (rho + 1e-20) of the first quantity, with the left
    // neighbour's density slope
    double W[E], WL, WR;
#pragma unroll
    for (int e = 0; e < E; e++) W[e] = fb_quot(q0[0][e], den[e], rden[e]);
    double DRL;
    {
      const double sL[2] = {W[E - 1], DR[E - 1]}, sR[1] = {W[0]};
      double xl[2], xr[1];
      AZR_X(2, 1, sL, xl, sR, xr);
      WL = xl[0];
      DRL = xl[1];
      WR = xr[0];
    }
    double RS[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const double ru = upl[e] ? ((e == 0) ? rL[0] : q0[RH][e - 1]) : q0[RH][e];
      const double du = upl[e] ? ((e == 0) ? DRL : DR[e - 1]) : DR[e];
      RS[e] = ru + f[e] * du;
    }
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      // van Leer slopes of the quotients (ComputeStarTheta)
      double D[E];
#pragma unroll
      for (int e = 0; e < E; e++) {
        const double wm = (e == 0) ? WL : W[e - 1], w0 = W[e], wp = (e == E - 1) ? WR : W[e + 1];
        const double dqm = (w0 - wm), dqp = (wp - w0);
        D[e] = fb_vl_slope(dqm, dqp, invdxtheta);
      }
      double DL;
      {
        const double sL[1] = {D[E - 1]};
        double xl[1];
        AZR_X(1, 0, sL, xl, sL, xl);
        DL = xl[0];
      }
      // star value and flux at each own lower face (VanLeerTheta)
      double F[E];
#pragma unroll
      for (int e = 0; e < E; e++) {
        const double ws = upl[e] ? ((e == 0) ? WL : W[e - 1]) : W[e];
        const double ds = upl[e] ? ((e == 0) ? DL : D[e - 1]) : D[e];
        const double qs = ws + f[e] * ds;
        F[e] = dxrad * qs * RS[e] * V[e];
      }
      // the next quantity's quotients travel with this one's first flux
      double Wn[E], WnL = 0.0, WnR = 0.0, FR;
      if (q + 1 < NQ) {
#pragma unroll
        for (int e = 0; e < E; e++) Wn[e] = fb_quot(q0[(q + 1 < NQ) ? q + 1 : q][e], den[e], rden[e]);
        const double sL[1] = {Wn[E - 1]}, sR[2] = {F[0], Wn[0]};
        double xl[1], xr[2];
        AZR_X(1, 2, sL, xl, sR, xr);
        FR = xr[0];
        WnR = xr[1];
        WnL = xl[0];
      } else {
        const double sR[1] = {F[0]};
        double xr[1];
        AZR_X(0, 1, sR, xr, sR, xr);
        FR = xr[0];
      }
#pragma unroll
      for (int e = 0; e < E; e++) {
        const double Fh = (e == E - 1) ? FR : F[e + 1];
        double varq = F[e];
        varq -= Fh;
        q0[q][e] = q0[q][e] + varq * invsurf;
      }
      if (q + 1 < NQ) {
#pragma unroll
        for (int e = 0; e < E; e++) W[e] = Wn[e];
        WL = WnL;
        WR = WnR;
      }
    }
  }
  // AdvectSHIFT (TransportEuler.c:350-373): cell c goes to c + nshift (mod
  // ns); ComputeVelocities' vtheta (TransportEuler.c:515-547) from the
  // pre-shift neighbours, floors on energy, sub-Keplerian edges
  int shift = (int)(nshift % ns);
  if (shift < 0) shift += ns;
  double xl[2];
  {
    const double sL[2] = {q0[2][E - 1], q0[RH][E - 1]};  // ThetaMomP and the density of the cell before
    AZR_X(2, 0, sL, xl, sL, xl);
  }
#undef AZR_X
  const int subkep = (!k.transport_only) && (i == 0 || i == nr - 1);
  const double rmi = tb.rmed;
#pragma unroll
  for (int e = 0; e < E; e++) {
    int p;
    if (TILE) {
      int g = (c0 + e) % ns;
      if (g < 0) g += ns;
      p = g + shift;
    } else {
      p = c0 + e + shift;
    }
    if (p >= ns) p -= ns;
    const double tpm = (e == 0) ? xl[0] : q0[2][e - 1], rm = (e == 0) ? xl[1] : q0[RH][e - 1];
    double v = (tpm + q0[3][e]) / (q0[RH][e] + rm + 1e-20) / rmi - rmi * omf(k);
    if (subkep) v = tb.vthetamed - rmi * omf(k);
    double en = 0.0;
    if (NQ == 6) {
      en = q0[(NQ == 6) ? 4 : 0][e];
      if (k.add_floors && !k.transport_only) {
        double e_bottom = 1e-3 * tb.energymed;
        if (en < e_bottom) en = e_bottom;
      }
    }
    out(e, p, v, q0[RH][e], q0[0][e], q0[1][e], en);
  }
}

template <int NQ, int E, int MT>
__global__ void __launch_bounds__(MT) k_transport_azimuthal_reg(KP k, double dtov)
{
  fb_grid_dependency();
  __shared__ double sh[32];
  __shared__ double hal[2][2][AZR_MAXW][AZR_NV];  // [buffer][0 last cells, 1 first cells][warp][value]
  const double dt = dt_of(k, dtov);
  const int i = blockIdx.x, ns = k.ns, T = blockDim.x, tid = threadIdx.x;
  const size_t base = (size_t)i * ns;
  const int c0 = tid * E;
  int xb = 0;
  // every global load at once: the own cells' quantities and vtheta, and
  // vtheta of the cells the ring mean of the other variants gives this thread
  double q0[NQ][E], vt[E], vs[E];
#pragma unroll
  for (int q = 0; q < NQ; q++) azr_load<E>(k.q[q] + base + c0, q0[q]);
  azr_load<E>(k.vt + base + c0, vt);
#pragma unroll
  for (int e = 0; e < E; e++) vs[e] = k.vt[base + tid + e * T];
  const AzrTab tb = azr_tab(k, i);
  azr_ring<NQ, E, false>(k, dt, i, tb, q0, vt, vs, 0.0, c0, sh, hal, xb,
                         [&](int, int p, double v, double r, double a, double b, double en) {
                    k.vt[base + p] = v;
                    k.rho_t[base + p] = r;
                    k.q[0][base + p] = a;
                    k.q[1][base + p] = b;
                    if (NQ == 6) k.e[base + p] = en;
                  });
}

// Tile variant of the azimuthal pass (variant 6): the register variant's
// arithmetic with no barrier.  A ring is cut into tiles of AZT_CO(E) = 32 E -
// 9 cells, one warp each (AZT_WPC warps of any rings per CTA).  A warp loads
// 32 E consecutive cells, the tile with 5 cells before it and 4 after, and
// advances all of them: a van Leer pass changes a cell from its neighbours
// up to two cells away, so after the residual and the uniform pass the
// cells 4 .. 32 E - 5 are exact, and ComputeVelocities' vtheta, which reads
// the cell before, is exact on the 32 E - 9 cells from the sixth on.  The
// halo costs 9 / (32 E) of redundant arithmetic; in exchange every
// neighbour value moves by a warp shuffle and the warps of an SM run
// independently.  Tiles of one ring run in different CTAs, so the pass
// cannot work in place: the radial pass leaves RadMomP, RadMomM and a copy
// of vtheta in three scratch fields (azt_buf) and this pass writes the usual
// outputs.  The ring mean of vtheta comes from k_azi_vmed, summed in the
// order of the register variant's CTA of azi_threads_for(nsec, E) threads,
// so for the same E the results agree to the last bit.
#define AZT_WPC 4
#define AZT_LEFT 5
#define AZT_HALO 9
#define AZT_CO(E) (32 * (E) - AZT_HALO)

__global__ void __launch_bounds__(1024) k_azi_vmed(KP k, double dtov)
{
  fb_grid_dependency();
  __shared__ double sh[32];
  const double dt = dt_of(k, dtov);
  const int i = blockIdx.x, ns = k.ns, T = blockDim.x;
  const double *vt = k.vt + (size_t)i * ns;
  const double invdt = 1.0 / dt;
  double s = 0.0;
  for (int j = threadIdx.x; j < ns; j += T) {
    double elong = vt[j] * dt;
    s += elong * invdt;
  }
  s = block_sum_dyn(s, sh);
  if (threadIdx.x == 0) k.azt_vmed[i] = s / (double)ns;
}

template <int NQ, int E, int MINB>
__global__ void __launch_bounds__(AZT_WPC * 32, MINB) k_transport_azimuthal_tile(KP k, double dtov)
{
  fb_grid_dependency();
  const double dt = dt_of(k, dtov);
  const int ns = k.ns;
  constexpr int CO = AZT_CO(E);
  const int ntiles = (ns + CO - 1) / CO;
  const int gw = blockIdx.x * AZT_WPC + (threadIdx.x >> 5);
  if (gw >= k.nr * ntiles) return;  // the whole warp
  const int i = gw / ntiles, t = gw - i * ntiles;
  const int lane = threadIdx.x & 31;
  const size_t base = (size_t)i * ns;
  const int c0 = t * CO - AZT_LEFT + lane * E;
  double q0[NQ][E], vt[E], vs[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    int g = (c0 + e) % ns;
    if (g < 0) g += ns;
    const size_t l = base + g;
#pragma unroll
    for (int q = 0; q < NQ; q++) q0[q][e] = (q < 2 ? k.azt_buf[q] : k.q[q])[l];
    vt[e] = k.azt_buf[2][l];
    vs[e] = 0.0;
  }
  const AzrTab tb = azr_tab(k, i);
  const double vmed = k.azt_vmed[i];
  int xb = 0;
  const int m0 = lane * E - AZT_LEFT, tcell = t * CO;  // tile cell of own cell e: m0 + e
  azr_ring<NQ, E, true>(k, dt, i, tb, q0, vt, vs, vmed, c0, nullptr, nullptr, xb,
                        [&](int e, int p, double v, double r, double a, double b, double en) {
                          const int m = m0 + e;
                          if (m < 0 || m >= CO || tcell + m >= ns) return;
                          k.vt[base + p] = v;
                          k.rho_t[base + p] = r;
                          k.q[0][base + p] = a;
                          k.q[1][base + p] = b;
                          if (NQ == 6) k.e[base + p] = en;
                        });
}

// Staged variant of the azimuthal pass (variant 5): the register variant's
// arithmetic in a persistent kernel (one CTA per SM, rings i = blockIdx.x,
// blockIdx.x + gridDim.x, ...).  A ring's NQ quantities and vtheta arrive in
// shared memory by bulk asynchronous copies (cp.async.bulk, completion on an
// mbarrier) issued one ring ahead, so the next ring's loads overlap this
// ring's arithmetic; the results are written back into the same buffer at
// their shifted cells and leave by bulk copies too, one contiguous row per
// field.  Two buffers of NQ + 1 rows of nsec doubles.  Every wait is bounded:
// a copy that never completes sets FB_ERR_TIMEOUT in the control block and the
// CTA stops.
static __device__ __forceinline__ unsigned azs_smem(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
static __device__ __forceinline__ void azs_expect(unsigned long long *bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(azs_smem(bar)), "r"(bytes)
               : "memory");
}
static __device__ __forceinline__ void azs_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   azs_smem(dst)),
               "l"(src), "r"(bytes), "r"(azs_smem(bar))
               : "memory");
}
static __device__ __forceinline__ void azs_store(void *dst, const void *src, unsigned bytes)
{
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(azs_smem(src)),
               "r"(bytes)
               : "memory");
}
// bounded wait for phase `parity` of the mbarrier: false after `limit` tries
static __device__ __forceinline__ bool azs_wait(unsigned long long *bar, unsigned parity, long long limit)
{
  for (long long it = 0; it < limit; it++) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(azs_smem(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
#define AZS_WAIT_LIMIT (1LL << 22)  // try_wait calls (each may suspend for a while): seconds, not forever

template <int NQ, int E, int MT>
__global__ void __launch_bounds__(MT) k_transport_azimuthal_staged(KP k, double dtov)
{
  fb_grid_dependency();
  extern __shared__ double2 azs_dyn[];
  __shared__ double sh[32];
  __shared__ double hal[2][2][AZR_MAXW][AZR_NV];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ int failed;
  const double dt = dt_of(k, dtov);
  const int ns = k.ns, nr = k.nr, T = blockDim.x, tid = threadIdx.x;
  const int c0 = tid * E;
  constexpr int NB = NQ + 1;  // rows per ring: the quantities and vtheta
  double *buf = (double *)azs_dyn;
  const unsigned row_bytes = (unsigned)ns * 8u;
  int xb = 0;
  // the rows of ring r into buffer b (one thread)
  auto issue = [&](int r, int b) {
    const size_t base = (size_t)r * ns;
    azs_expect(&bar[b], NB * row_bytes);
#pragma unroll
    for (int q = 0; q < NQ; q++) azs_load(buf + (size_t)(b * NB + q) * ns, k.q[q] + base, row_bytes, &bar[b]);
    azs_load(buf + (size_t)(b * NB + NQ) * ns, k.vt + base, row_bytes, &bar[b]);
  };
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(azs_smem(&bar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(azs_smem(&bar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    failed = 0;
    if ((int)blockIdx.x < nr) issue(blockIdx.x, 0);
  }
  __syncthreads();
  int it = 0;
  for (int i = blockIdx.x; i < nr; i += gridDim.x, it++) {
    const int b = it & 1;
    const size_t base = (size_t)i * ns;
    const AzrTab tb = azr_tab(k, i);  // in flight while the copies complete
    // the next ring into the other buffer, once the bulk stores of the ring
    // it held last have read it
    if (tid == 0 && i + (int)gridDim.x < nr) {
      asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      issue(i + gridDim.x, b ^ 1);
    }
    if (!azs_wait(&bar[b], (unsigned)((it >> 1) & 1), AZS_WAIT_LIMIT)) failed = 1;
    __syncthreads();
    if (failed) break;
    const double *rows = buf + (size_t)b * NB * ns;
    double q0[NQ][E], vt[E], vs[E];
#pragma unroll
    for (int q = 0; q < NQ; q++)
#pragma unroll
      for (int e = 0; e < E; e++) q0[q][e] = rows[(size_t)q * ns + c0 + e];
#pragma unroll
    for (int e = 0; e < E; e++) {
      vt[e] = rows[(size_t)NQ * ns + c0 + e];
      vs[e] = rows[(size_t)NQ * ns + tid + e * T];
    }
    __syncthreads();  // every row read: the buffer takes the results
    double *o = buf + (size_t)b * NB * ns;
    azr_ring<NQ, E, false>(k, dt, i, tb, q0, vt, vs, 0.0, tid * E, sh, hal, xb,
                           [&](int, int p, double v, double r, double a, double bb, double en) {
                      o[p] = v;
                      o[(size_t)ns + p] = r;
                      o[(size_t)2 * ns + p] = a;
                      o[(size_t)3 * ns + p] = bb;
                      if (NQ == 6) o[(size_t)4 * ns + p] = en;
                    });
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the results, visible to the bulk copies
    __syncthreads();
    if (tid == 0) {
      azs_store(k.vt + base, o, row_bytes);
      azs_store(k.rho_t + base, o + ns, row_bytes);
      azs_store(k.q[0] + base, o + (size_t)2 * ns, row_bytes);
      azs_store(k.q[1] + base, o + (size_t)3 * ns, row_bytes);
      if (NQ == 6) azs_store(k.e + base, o + (size_t)4 * ns, row_bytes);
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
  }
  if (tid == 0) {
    if (failed) {
      k.ctl->status = FB_ERR_TIMEOUT;
      // a load still in flight lands in this CTA's buffer: give it a bounded
      // time to arrive before the CTA's shared memory goes away
      azs_wait(&bar[it & 1], (unsigned)((it >> 1) & 1), AZS_WAIT_LIMIT);
    }
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // the results are in global memory
  }
}

// cells per thread of the azimuthal pass (1..4): at most 1024 threads for
// 1-2 cells each, 768 threads for 3-4 (more registers per thread).  The
// automatic choice is the fewest cells per thread; the tuner may pick more.
static int azi_max_threads(int E) { return E <= 2 ? 1024 : 768; }
static int azi_threads_for(int ns, int E) { return (((ns + E - 1) / E) + 31) / 32 * 32; }
int fb_azi_E_auto(int ns)
{
  for (int E = 1; E <= 4; E++)
    if (azi_threads_for(ns, E) <= azi_max_threads(E)) return E;
  return 5;  // ring too long
}
static int max_smem_optin()
{
  int dev = 0, maxopt = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return maxopt;
}
int fb_azi_E_valid(int ns, int energy, int E)
{
  if (E < 1 || E > 4 || azi_threads_for(ns, E) > azi_max_threads(E)) return 0;
  const int NQ = energy ? 6 : 5;
  return (size_t)FB_AZI_RINGS(NQ) * ns * sizeof(double) + 32 * sizeof(double) <= (size_t)max_smem_optin();
}
// Variants of the azimuthal pass: 1 narrow, 2 wide, 3 packed.  The wide and
// packed ones need their rings to fit and at most 768 threads for two or
// more cells per thread; variant 0 takes the packed one, else the wide one,
// else the narrow one.  Returns the variant a launch takes, 0 if `variant`
// cannot run on this ring.
static bool azi_fits(int ns, int E, size_t rings)
{
  const int maxt = (E == 1) ? 1024 : 768;
  return azi_threads_for(ns, E) <= maxt &&
         rings * ns * sizeof(double) + 32 * sizeof(double) <= (size_t)max_smem_optin();
}
// The register variant needs E >= 2 contiguous cells per thread with
// nsec = E T, T a multiple of 32 within the kernel's thread limit.
static bool azr_fits(int ns, int E)
{
  if (E < 2 || E > 4 || ns % E != 0) return false;
  const int T = ns / E;
  return T % 32 == 0 && T <= AZR_MAXT && T / 32 <= AZR_MAXW;
}
// The staged variant: two buffers of NQ + 1 rows of nsec doubles, rows of a
// whole number of 16-byte units (even nsec), 16-byte aligned fields.
static size_t azs_smem_bytes(int ns, int NQ) { return (size_t)2 * (NQ + 1) * ns * sizeof(double); }
static bool azs_fits(int ns, int energy, int E)
{
  const int NQ = energy ? 6 : 5;
  return azr_fits(ns, E) && ns % 2 == 0 &&
         azs_smem_bytes(ns, NQ) + 4096 <= (size_t)max_smem_optin();
}
static bool azs_pointers_aligned(const KP &k, int NQ)
{
  auto al = [](const void *p) { return ((unsigned long long)p & 15ull) == 0; };
  bool ok = al(k.vt) && al(k.rho_t) && (NQ != 6 || al(k.e));
  for (int q = 0; q < NQ; q++) ok = ok && al(k.q[q]);
  return ok;
}
// one CTA per ring up to the CTAs the GPU holds at once
static int azs_grid(const void *fn, int threads, size_t smem, int nr)
{
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int g = sms * per_sm;
  return g < nr ? g : nr;
}
// The tile variant: 2 to 4 cells per lane, and the ring-mean kernel's CTA
// of azi_threads_for(nsec, E) threads within 1024.
static bool azt_fits(int ns, int E) { return E >= 2 && E <= 4 && azi_threads_for(ns, E) <= 1024; }
int fb_azi_variant(int ns, int energy, int E, int variant)
{
  const int NQ = energy ? 6 : 5;
  const bool wide = azi_fits(ns, E, FB_AZI_RINGS_WIDE(NQ)), packed = azi_fits(ns, E, AZP_RINGS(NQ));
  switch (variant) {
    case 0: return packed ? 3 : wide ? 2 : 1;
    case 1: return 1;
    case 2: return wide ? 2 : 0;
    case 3: return packed ? 3 : 0;
    case 4: return azr_fits(ns, E) ? 4 : 0;
    case 5: return azs_fits(ns, energy, E) ? 5 : 0;
    case 6: return azt_fits(ns, E) ? 6 : 0;
    case 7: return azt_fits(ns, E) ? 7 : 0;
    case 8: return azt_fits(ns, E) ? 8 : 0;
    default: return 0;
  }
}
// The variant and cells per thread a launch of this KP's azimuthal pass
// takes: the tuned ones where they can run, the staged variant only on
// 16-byte aligned fields, the tile variant only with its scratch fields.
static int azi_resolve(const KP &k, int *Eout)
{
  const int NQ = k.energy ? 6 : 5;
  const int E = k.azi_E > 0 ? k.azi_E : fb_azi_E_auto(k.ns);
  int var = fb_azi_variant(k.ns, k.energy, E, k.azi_variant);
  if (var == 0) var = 1;
  if (var == 5 && !azs_pointers_aligned(k, NQ)) var = 4;  // bulk copies need 16-byte aligned rows
  if ((var == 6 || var == 7 || var == 8) && !(k.azt_buf[0] && k.azt_buf[1] && k.azt_buf[2] && k.azt_vmed))
    var = azr_fits(k.ns, E) ? 4 : 1;
  if (Eout) *Eout = E;
  return var;
}
static bool azt_variant(int var) { return var == 6 || var == 7 || var == 8; }
int fb_azi_launches(const KP &k) { return azt_variant(azi_resolve(k, nullptr)) ? 2 : 1; }

// LostMass += LostByDisk of the density's VanLeerRadial (TransportEuler.c:137,
// :213-216): the ring-0 radial fluxes summed over azimuth by one warp, lane
// by lane in azimuth order, then across lanes; a batch's loads all in flight.
static __device__ __forceinline__ void lost_mass_sum(const KP &k)
{
  constexpr int U = 24;  // 1536 azimuths: two batches
  double s = 0.0;
  for (int j0 = threadIdx.x; j0 < k.ns; j0 += 32 * U) {
    double v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int j = j0 + 32 * u;
      v[u] = (j < k.ns) ? k.lost0[j] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; u++)
      if (j0 + 32 * u < k.ns) s += v[u];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) k.ctl->lost_mass += 0.0 + s;
}

// ComputeVelocities' radial part (TransportEuler.c:531-536) needs the
// neighbouring ring after both passes; fused with AddFloorDensity
// (SourceEuler.c:2506) and ApplyWallBoundaries (SideEuler.c:1047-1099).
// The first warp of the first CTA also adds the lost mass.
__global__ void __launch_bounds__(FB_BS2) k_transport_vr(KP k)
{
  fb_grid_dependency();
  const int ns = k.ns, nr = k.nr;
  const int wall = k.wall && !k.transport_only;
  const int floors = k.add_floors && !k.transport_only;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x < 32) lost_mass_sum(k);
  {
    const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    const size_t l = (size_t)i * ns + j;
    auto vr_at = [&](int ii) -> double {
      if (ii == 0) return 0.0;
      const size_t m = (size_t)ii * ns + j;
      return (k.q[0][m - ns] + k.q[1][m]) / (k.rho_t[m] + k.rho_t[m - ns] + 1e-20);
    };
    if (i == nr) {
      if (wall) k.vr[l] = -vr_at(nr - 2);
      return;
    }
    double d = k.rho_t[l];
    double v = vr_at(i);
    if (floors && d < k.floordens) d = k.floordens;
    if (wall) {
      if (i == 1) { v = 0.0; d = k.sigmamed[1]; }
      if (i == 0) { v = -vr_at(2); d = k.sigmamed[0]; }
      if (i == nr - 1) { v = 0.0; d = k.sigmamed[nr - 1]; }
      if (i == nr - 2) d = k.sigmamed[nr - 2];
    }
    k.rho[l] = d;
    k.vr[l] = v;
  }
}

// Ring chunks of the radial pass that fill whole waves: for r = 1..6 rounds
// of the CTAs the GPU holds at once (`tx` columns per CTA), the smallest
// chunk whose grid takes at most r rounds.  A CTA's time grows with its
// chunk plus the two halo rings it rereads, so a grid one CTA past a wave
// costs a whole extra round; these chunks avoid that.  Returns how many
// were written to out (increasing r, decreasing chunk).
// CTAs of the radial pass (2 tx threads) the GPU holds at once, 0 if unknown.
static int rad_resident_ctas(int energy, int tx)
{
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 0;
  const cudaError_t e = energy ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_transport_radial<6>, 2 * tx, 0)
                               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_transport_radial<5>, 2 * tx, 0);
  if (e != cudaSuccess || per < 1 || sms < 1) {
    cudaGetLastError();
    return 0;
  }
  return per * sms;
}

int fb_rad_chunks_balanced(const KP &k, int tx, int *out, int max)
{
  const int slots = rad_resident_ctas(k.energy, tx);
  if (slots < 1) return 0;
  const int bx = (k.ns + tx - 1) / tx;
  int n = 0;
  for (int r = 1; r <= 6 && n < max; r++) {
    const int rows = (r * slots) / bx;  // ring chunks that r rounds hold
    if (rows < 1) continue;
    int ch = (k.nr + rows - 1) / rows;
    if (ch < 2) ch = 2;
    if (n == 0 || out[n - 1] != ch) out[n++] = ch;
  }
  return n;
}

// Rings per CTA of the radial pass when not tuned: 64-column CTAs and, of
// the wave-filling chunks, the one with the least rounds x (chunk + 2 halo
// rings); 16 if the occupancy query fails.
int fb_rad_chunk_auto(const KP &k)
{
  const int tx = k.rad_tx > 0 ? k.rad_tx : 64;
  int ch[6];
  const int n = fb_rad_chunks_balanced(k, tx, ch, 6);
  if (n == 0) return 16;
  const int bx = (k.ns + tx - 1) / tx;
  const long slots = rad_resident_ctas(k.energy, tx);
  int best = ch[0];
  long bestcost = -1;
  for (int q = 0; q < n; q++) {
    const long ctas = (long)bx * ((k.nr + ch[q] - 1) / ch[q]);
    const long rounds = (ctas + slots - 1) / slots;
    const long cost = rounds * (ch[q] + 2);
    if (bestcost < 0 || cost < bestcost) { bestcost = cost; best = ch[q]; }
  }
  return best;
}

void fb_launch_transport_radial(const KP &k0, double dt_override, cudaStream_t s)
{
  // before the tile variant: RadMomP, RadMomM and a copy of vtheta into its
  // scratch fields (it cannot update them in place)
  KP k = k0;
  k.vt_copy = nullptr;
  if (azt_variant(azi_resolve(k0, nullptr))) {
    k.q[0] = k0.azt_buf[0];
    k.q[1] = k0.azt_buf[1];
    k.vt_copy = k0.azt_buf[2];
  }
  const int tx = k.rad_tx > 0 ? k.rad_tx : 64, bx = (k.ns + tx - 1) / tx;
  const int chunk = k.rad_chunk > 0 ? k.rad_chunk : fb_rad_chunk_auto(k);
  dim3 gr(bx, (k.nr + chunk - 1) / chunk);
  if (k.energy)
    fb_launch(k_transport_radial<6>, gr, 2 * tx, 0, s, k, dt_override, chunk);
  else
    fb_launch(k_transport_radial<5>, gr, 2 * tx, 0, s, k, dt_override, chunk);
}

// The tile variant's ring means of vtheta (k_azi_vmed): nothing between
// SubStep2 and the azimuthal pass changes vtheta, so the step may run them
// on a branch beside SubStep3 and the radial pass.  Returns the launches.
int fb_launch_azi_vmed(const KP &k, double dt_override, cudaStream_t s)
{
  int E = 1;
  if (!azt_variant(azi_resolve(k, &E))) return 0;
  fb_launch(k_azi_vmed, k.nr, azi_threads_for(k.ns, E), 0, s, k, dt_override);
  return 1;
}

template <int NQ>
static void launch_azimuthal(const KP &k, double dt_override, cudaStream_t s, bool vmed_done)
{
  int E = 1;
  const int var = azi_resolve(k, &E);
  const bool wide = (var == 2);
  const int th = azi_threads_for(k.ns, E);
  const bool full = (th * E == k.ns);  // every thread owns E cells
  if (var == 6 || var == 7 || var == 8) {
    if (!vmed_done) fb_launch(k_azi_vmed, k.nr, th, 0, s, k, dt_override);
    const int CO = AZT_CO(E), ntiles = (k.ns + CO - 1) / CO;
    const int grid = (int)(((long)k.nr * ntiles + AZT_WPC - 1) / AZT_WPC);
#define AZT_LAUNCH(EE, MB) fb_launch(k_transport_azimuthal_tile<NQ, EE, MB>, grid, AZT_WPC * 32, 0, s, k, dt_override)
    if (var == 6) {
      switch (E) {
        case 2: AZT_LAUNCH(2, 4); break;
        case 3: AZT_LAUNCH(3, 4); break;
        default: AZT_LAUNCH(4, 4); break;
      }
    } else if (var == 8) {  // five CTAs per SM (at most 102 registers)
      switch (E) {
        case 2: AZT_LAUNCH(2, 5); break;
        case 3: AZT_LAUNCH(3, 5); break;
        default: AZT_LAUNCH(4, 5); break;
      }
    } else {
      switch (E) {
        case 2: AZT_LAUNCH(2, 3); break;
        case 3: AZT_LAUNCH(3, 3); break;
        default: AZT_LAUNCH(4, 3); break;
      }
    }
#undef AZT_LAUNCH
    return;
  }
  if (var == 5) {
    const int T = k.ns / E;
    const size_t smem = azs_smem_bytes(k.ns, NQ);
#define AZS_LAUNCH(EE, MM)                                                                                \
  fb_launch(k_transport_azimuthal_staged<NQ, EE, MM>,                                                   \
            azs_grid((const void *)k_transport_azimuthal_staged<NQ, EE, MM>, MM, smem, k.nr), T, smem, s, k, \
            dt_override)
#define AZS_E(EE)                                                                                   \
  (T <= 256 ? AZS_LAUNCH(EE, 256) : T <= 384 ? AZS_LAUNCH(EE, 384) : T <= 512 ? AZS_LAUNCH(EE, 512)  \
                                                                   : AZS_LAUNCH(EE, 768))
    switch (E) {
      case 2: AZS_E(2); break;
      case 3: AZS_E(3); break;
      default: AZS_E(4); break;
    }
#undef AZS_E
#undef AZS_LAUNCH
    return;
  }
  if (var == 4) {
    // the instance bounded by the smallest of 256 / 384 / 512 / 768 threads
    // that holds T: the fewer threads, the more registers each may use
    const int T = k.ns / E;
#define AZR_LAUNCH(EE)                                                                                   \
  (T <= 256 ? fb_launch(k_transport_azimuthal_reg<NQ, EE, 256>, k.nr, T, 0, s, k, dt_override)            \
   : T <= 384 ? fb_launch(k_transport_azimuthal_reg<NQ, EE, 384>, k.nr, T, 0, s, k, dt_override)          \
   : T <= 512 ? fb_launch(k_transport_azimuthal_reg<NQ, EE, 512>, k.nr, T, 0, s, k, dt_override)          \
              : fb_launch(k_transport_azimuthal_reg<NQ, EE, 768>, k.nr, T, 0, s, k, dt_override))
    switch (E) {
      case 2: AZR_LAUNCH(2); break;
      case 3: AZR_LAUNCH(3); break;
      default: AZR_LAUNCH(4); break;
    }
#undef AZR_LAUNCH
    return;
  }
  if (var == 3) {
    const size_t psmem = (size_t)AZP_RINGS(NQ) * k.ns * sizeof(double);
#define AZP_LAUNCH(EE)                                                                                       \
  (full ? fb_launch(k_transport_azimuthal_packed<NQ, EE, true>, k.nr, th, psmem, s, k, dt_override)           \
        : fb_launch(k_transport_azimuthal_packed<NQ, EE, false>, k.nr, th, psmem, s, k, dt_override))
    switch (E) {
      case 1: AZP_LAUNCH(1); break;
      case 2: AZP_LAUNCH(2); break;
      case 3: AZP_LAUNCH(3); break;
      default: AZP_LAUNCH(4); break;
    }
#undef AZP_LAUNCH
    return;
  }
  const size_t smem = (size_t)(wide ? FB_AZI_RINGS_WIDE(NQ) : FB_AZI_RINGS(NQ)) * k.ns * sizeof(double);
#define AZI_LAUNCH(EE)                                                                                     \
  (wide ? (full ? fb_launch(k_transport_azimuthal<NQ, EE, true, true>, k.nr, th, smem, s, k, dt_override)         \
                : fb_launch(k_transport_azimuthal<NQ, EE, false, true>, k.nr, th, smem, s, k, dt_override))       \
        : (full ? fb_launch(k_transport_azimuthal<NQ, EE, true, false>, k.nr, th, smem, s, k, dt_override)        \
                : fb_launch(k_transport_azimuthal<NQ, EE, false, false>, k.nr, th, smem, s, k, dt_override)))
  switch (E) {
    case 1: AZI_LAUNCH(1); break;
    case 2: AZI_LAUNCH(2); break;
    case 3: AZI_LAUNCH(3); break;
    default: AZI_LAUNCH(4); break;
  }
#undef AZI_LAUNCH
}

void fb_launch_transport_azimuthal(const KP &k, double dt_override, cudaStream_t s, bool vmed_done)
{
  if (k.energy)
    launch_azimuthal<6>(k, dt_override, s, vmed_done);
  else
    launch_azimuthal<5>(k, dt_override, s, vmed_done);
}

void fb_launch_transport_vr(const KP &k, cudaStream_t s)
{
  fb_launch(k_transport_vr, grid2d(k, k.nr + 1), k.cell_bs, 0, s, k);
}

// ------------------------------------------- open and non-reflecting edges
// ApplyBoundaryCondition's edges other than the wall (SideEuler.c:1102-1131),
// after the transport and floors and before the damping, as AlgoGas calls it
// (SourceEuler.c:695): OpenBoundary (SideEuler.c:300-410; with INNERBOUNDARY
// K, Kley & Nelson's outflow of :325-338) and NonReflectingBoundary
// (SideEuler.c:569-794).  One CTA per edge: blockIdx.x 0 the inner edge, 1 the
// outer.  The ring means the non-reflecting edge takes are summed by one
// fixed tree (the reference sums sequentially: ~1e-16 relative).  Where the
// reference leaves the innermost (outermost) planet's radius undefined (no
// planet inside the grid), the planets' frequency term is 0 here.
#define EDGE_BS 256
__global__ void __launch_bounds__(EDGE_BS) k_edges(KP k)
{
  fb_grid_dependency();
  __shared__ double sh[32];
  const int ns = k.ns, nr = k.nr, tid = threadIdx.x, T = blockDim.x;
  const bool inner = (blockIdx.x == 0);
  double *rho = k.rho, *vr = k.vr, *vt = k.vt, *en = k.e;
  const double *cs = k.cs;
  if (k.open_inner) {
    if (inner) {
      const int i = 2;
      for (int j = tid; j < ns; j += T) {
        const size_t l = (size_t)j + (size_t)i * ns;
        if (k.kn_open) {
          rho[l - ns] = rho[l] * k.rmed[1] / k.rmed[0];
          if (k.energy) en[l - ns] = en[l];
          if (vr[l + ns] > 0.0) {
            vr[l] = 0.0;
          } else {
            const double vri = -3. * nu_ring(k, i) / k.rmed[i] * 3. * (-k.sigmaslope + 1. + 2. * k.flaringindex);
            if (fabs(vr[l + ns]) > fabs(vri))
              vr[l] = vri;
            else
              vr[l] = vr[l + ns];
          }
        } else {
          rho[l - ns] = rho[l];
          rho[l - 2 * ns] = rho[l];
          if (k.energy) {
            en[l - ns] = en[l];
            en[l - 2 * ns] = en[l];
          }
          vt[l - ns] = vt[l] * k.ob_vt1;
          vt[l - 2 * ns] = vt[l] * k.ob_vt0;
          if ((vr[l + ns] >= 0.0) || (rho[l] < k.sigmamed[0])) {
            vr[l] = 0.0;
            vr[l - ns] = 0.0;
          } else {
            vr[l] = vr[l + ns];
            vr[l - ns] = vr[l + ns];
          }
        }
      }
    } else {
      const int i = nr - 1;
      for (int j = tid; j < ns; j += T) {
        const size_t l = (size_t)j + (size_t)i * ns;
        rho[l] = rho[l - ns];
        if (k.energy) en[l] = en[l - ns];
        vt[l] = vt[l - ns] * k.ob_vtout;
        if (k.kn_open) {
          if (vr[l - ns] < 0.0)
            vr[l] = 0.0;
          else
            vr[l] = vr[l - ns];
        } else {
          if ((vr[l - ns] < 0.0) || (rho[l] < k.sigmamed[nr - 2]))
            vr[l] = 0.0;
          else
            vr[l] = vr[l - ns];
        }
      }
    }
  }
  if (!k.non_reflecting) return;
  const fb_ctl *c = k.ctl;
  if (inner) {
    // innermost planet inside the grid (SideEuler.c:589-599)
    double buf = k.radiin, omega_in = 0.0;
    for (int q = 0; q < c->np; q++) {
      const double rp = sqrt(c->px[q] * c->px[q] + c->py[q] * c->py[q]);
      if ((rp < buf) && (rp >= k.radii0)) {
        buf = rp;
        omega_in = pow(rp, -1.5);
      }
    }
    const int i = 1;
    // the ring means and the shift (SideEuler.c:607-626 isothermal,
    // :662-674 adiabatic)
    double cs1 = 0.0, d1 = 0.0, dangle;
    if (!k.energy) {
      double cs0 = 0.0, d0 = 0.0;
      for (int j = tid; j < ns; j += T) {
        cs0 += cs[j];
        cs1 += cs[ns + j];
        d0 += rho[j];
        d1 += rho[ns + j];
      }
      cs0 = block_sum_dyn(cs0, sh) / (double)ns;
      cs1 = block_sum_dyn(cs1, sh) / (double)ns;
      d0 = block_sum_dyn(d0, sh) / (double)ns;  // dens0: unused without an accreting edge
      d1 = block_sum_dyn(d1, sh) / (double)ns;
      (void)d0;
      dangle = (k.nrb_om1 - omega_in) / (.5 * (cs0 + cs1));
    } else {
      dangle = (k.nrb_om1 - omega_in) / (.5 * (k.nrb_csinit0 + k.nrb_csinit1));
    }
    dangle *= (k.rmed[1] - k.rmed[0]);
    const int i_angle = (int)(dangle / (k.pmax - k.pmin) * (double)ns + .5);
    // The reference's loop copies ring 1 into ring 0 shifted by i_angle
    // cells, wrapping once: a shift beyond one turn writes cells of ring 1
    // the loop has already read (the same values result when every read is
    // done before any write).  A shift beyond two turns, or one that writes
    // below ring 0, is not reproduced: the DT stops with
    // FB_ERR_UNSUPPORTED.  The density (isothermal) or the energy
    // (adiabatic) is copied; vrad from the old density of ring 1.
    double *f = k.energy ? en : rho, *ebuf = k.edge_buf;
    int bad = 0;
    for (int j = tid; j < ns; j += T) {
      const size_t l = (size_t)j + (size_t)i * ns;
      int jp = j + i_angle;
      if (jp >= ns) jp -= ns;
      if (jp < 0) jp += ns;
      if (jp < 0 || jp >= 2 * ns || (jp >= ns && jp - ns > j)) bad = 1;
      ebuf[j] = f[l];
      const double vr_med = k.energy ? -k.nrb_csinit1 * (rho[l] - k.sigmamed[1]) / k.sigmamed[1]
                                     : -cs1 * (rho[l] - d1) / d1;
      vr[l] = 2. * vr_med - vr[l + ns];
    }
    if (__syncthreads_or(bad)) {
      if (tid == 0) k.ctl->status = FB_ERR_UNSUPPORTED;
      return;
    }
    for (int j = tid; j < ns; j += T) {
      int jp = j + i_angle;
      if (jp >= ns) jp -= ns;
      if (jp < 0) jp += ns;
      f[jp] = ebuf[j];
    }
    __syncthreads();
    if (!k.energy) {
      double mean = 0.0;
      for (int j = tid; j < ns; j += T) mean += rho[j];
      mean = block_sum_dyn(mean, sh) / (double)ns;
      for (int j = tid; j < ns; j += T) rho[j] += (k.sigmamed[0] - mean);
    } else {
      const double csinit0 = k.nrb_csinit0;
      for (int j = tid; j < ns; j += T)
        rho[j] = k.sigmamed[0] + (k.gamma - 1.0) * (en[j] - k.energymed[0]) / csinit0 / csinit0;
      __syncthreads();
      double mean = 0.0;
      for (int j = tid; j < ns; j += T) mean += rho[j];
      mean = block_sum_dyn(mean, sh) / (double)ns;
      for (int j = tid; j < ns; j += T) rho[j] += (k.sigmamed[0] - mean);
      __syncthreads();
      mean = 0.0;
      for (int j = tid; j < ns; j += T) mean += en[j];
      mean = block_sum_dyn(mean, sh) / (double)ns;
      for (int j = tid; j < ns; j += T) en[j] += (k.energymed[0] - mean);
    }
  } else {
    // outermost planet inside the grid (SideEuler.c:718-728)
    double buf = k.radii0, omega_out = 0.0;
    for (int q = 0; q < c->np; q++) {
      const double rp = sqrt(c->px[q] * c->px[q] + c->py[q] * c->py[q]);
      if ((rp > buf) && (rp <= k.radiin)) {
        buf = rp;
        omega_out = pow(rp, -1.5);
      }
    }
    const int i = nr - 1;
    const size_t b1 = (size_t)(nr - 1) * ns, b2 = (size_t)(nr - 2) * ns;
    double c2 = 0.0, c1 = 0.0, d1 = 0.0, d2 = 0.0;
    for (int j = tid; j < ns; j += T) {
      c2 += cs[b2 + j];
      c1 += cs[b1 + j];
      d1 += rho[b1 + j];
      d2 += rho[b2 + j];
    }
    const double csnrm2 = block_sum_dyn(c2, sh) / (double)ns;
    const double csnrm1 = block_sum_dyn(c1, sh) / (double)ns;
    const double densnrm1 = block_sum_dyn(d1, sh) / (double)ns;  // unused without an accreting edge
    const double densnrm2 = block_sum_dyn(d2, sh) / (double)ns;
    (void)densnrm1;
    double dangle = (k.nrb_omn2 - omega_out) / (.5 * (csnrm1 + csnrm2));
    dangle *= (k.rmed[nr - 1] - k.rmed[nr - 2]);
    const int i_angle = (int)(dangle / (k.pmax - k.pmin) * (double)ns + .5);
    // The reference's loop sets cell j of ring nr-1 from cell j - i_angle of
    // ring nr-2, wrapping once: a shift beyond one turn reads cells of ring
    // nr-1 itself, the new value where the loop has already written the cell
    // (followed back to its own source), else the old one.  Every source is
    // resolved and read before any cell is written.  A source outside rings
    // 3 .. nr-1 is not reproduced (FB_ERR_UNSUPPORTED).
    double *bufr = k.edge_buf + ns, *bufe = k.edge_buf + 2 * (size_t)ns;
    int bad = 0;
    for (int j = tid; j < ns; j += T) {
      const size_t l = (size_t)j + b1;
      long src = -1;
      int jj = j;
      for (int it = 0; it <= ns; it++) {
        int jp = jj - i_angle;
        if (jp >= ns) jp -= ns;
        if (jp < 0) jp += ns;
        if (jp < ns) {
          src = (long)(i - 1) * ns + jp;
          break;
        }
        const int cc = jp - ns;  // a cell of ring nr-1
        if (cc >= ns) break;
        if (cc < jj) {
          jj = cc;
          continue;
        }
        src = (long)i * ns + cc;
        break;
      }
      if (src < 3L * ns || src >= (long)nr * ns) {
        bad = 1;
        src = (long)l;
      }
      bufr[j] = rho[src];
      bufe[j] = en[src];
      const double vr_med = (!k.energy) ? csnrm1 * (rho[l - ns] - densnrm2) / densnrm2
                                        : cs[l] * (rho[l - ns] - densnrm2) / densnrm2;
      vr[l] = 2. * vr_med - vr[l - ns];
    }
    if (__syncthreads_or(bad)) {
      if (tid == 0) k.ctl->status = FB_ERR_UNSUPPORTED;
      return;
    }
    for (int j = tid; j < ns; j += T) {
      rho[b1 + j] = bufr[j];
      en[b1 + j] = bufe[j];
    }
    __syncthreads();
    double mean = 0.0;
    for (int j = tid; j < ns; j += T) mean += rho[b1 + j];
    mean = block_sum_dyn(mean, sh) / (double)ns;
    for (int j = tid; j < ns; j += T) rho[b1 + j] += k.sigmamed[nr - 1] - mean;
    __syncthreads();
    mean = 0.0;
    for (int j = tid; j < ns; j += T) mean += en[b1 + j];
    mean = block_sum_dyn(mean, sh) / (double)ns;
    for (int j = tid; j < ns; j += T) en[b1 + j] += k.energymed[nr - 1] - mean;
  }
}

void fb_launch_edges(const KP &k, cudaStream_t s) { fb_launch(k_edges, 2, EDGE_BS, 0, s, k); }

// Makes the driver load the radial and vr transport kernels now (asking
// for a function's attributes loads it under lazy module loading), so that
// their first launch later needs no module load.  fb_gas_prepare does the
// same for every azimuthal variant.
int fb_transport_preload(void)
{
  const void *fns[] = {(const void *)k_transport_radial<5>, (const void *)k_transport_radial<6>,
                       (const void *)k_transport_vr};
  cudaFuncAttributes fa;
  for (const void *f : fns)
    if (cudaFuncGetAttributes(&fa, f) != cudaSuccess) return FB_ERR_CUDA;
  return FB_OK;
}

// Transport (TransportEuler.c:65-87) + floors + boundaries: 3 launches
void fb_launch_transport(const KP &k, double dt_override, cudaStream_t s)
{
  fb_launch_transport_radial(k, dt_override, s);
  fb_launch_transport_azimuthal(k, dt_override, s);
  fb_launch_transport_vr(k, s);
}

void fb_launch_floors_boundary(const KP &k, cudaStream_t s) { (void)k; (void)s; }

// ApplyBoundaryCondition alone (SideEuler.c:1102-1131): walls and the
// sub-Keplerian edge rings on the current state (stage tests).
__global__ void k_boundary_only(KP k)
{
  fb_grid_dependency();
  const int ns = k.ns, nr = k.nr;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  if (k.wall) {
    k.vr[(size_t)1 * ns + j] = 0.0;
    k.vr[j] = -k.vr[(size_t)2 * ns + j];
    k.rho[(size_t)1 * ns + j] = k.sigmamed[1];
    k.rho[j] = k.sigmamed[0];
    k.vr[(size_t)(nr - 1) * ns + j] = 0.0;
    k.vr[(size_t)nr * ns + j] = -k.vr[(size_t)(nr - 2) * ns + j];
    k.rho[(size_t)(nr - 2) * ns + j] = k.sigmamed[nr - 2];
    k.rho[(size_t)(nr - 1) * ns + j] = k.sigmamed[nr - 1];
  }
  k.vt[j] = k.vthetamed[0] - k.rmed[0] * omf(k);
  k.vt[(size_t)(nr - 1) * ns + j] = k.vthetamed[nr - 1] - k.rmed[nr - 1] * omf(k);
}

void fb_launch_boundary_only(const KP &k, cudaStream_t s)
{
  fb_launch(k_boundary_only, (k.ns + 127) / 128, 128, 0, s, k);
}

// ------------------------------------------------------------ damping
// EvanescentBoundary (SideEuler.c:796-950), default DampToAxi or DampToIni.
__global__ void __launch_bounds__(FB_BS) k_damping(KP k, double dtov)
{
  fb_grid_dependency();
  __shared__ double shm[4 * 32];
  const int i = k.damp_rings[blockIdx.x], ns = k.ns, nr = k.nr;
  const size_t base = (size_t)i * ns;
  const double step = dt_of(k, dtov);
  const double lambda = k.damp_lam[i] * step / k.damp_tau[i];
  double vrad0, vtheta0, dens0, energ0;
  if (k.damp_axi) {
    // the four ring means: each thread's partial sums in azimuth order (a
    // batch's loads in flight together), then one four-value tree, the same
    // order as four single sums
    double m[4] = {0.0, 0.0, 0.0, 0.0};
    for (int j0 = threadIdx.x; j0 < ns; j0 += RING_U * FB_BS) {
      double v[RING_U][4];
#pragma unroll
      for (int u = 0; u < RING_U; u++) {
        const int j = j0 + u * FB_BS;
        if (j < ns) {
          v[u][0] = k.vr[base + j];
          v[u][1] = k.vt[base + j];
          v[u][2] = k.rho[base + j];
          v[u][3] = k.e[base + j];
        }
      }
#pragma unroll
      for (int u = 0; u < RING_U; u++)
        if (j0 + u * FB_BS < ns) {
#pragma unroll
          for (int q = 0; q < 4; q++) m[q] += v[u][q];
        }
    }
    block_sums<4>(m, shm);
    vrad0 = m[0] / (double)ns;
    vtheta0 = m[1] / (double)ns;
    dens0 = m[2] / (double)ns;
    energ0 = m[3] / (double)ns;
  } else {
    vtheta0 = k.vthetamed[i] - k.rmed[i] * omf(k);
    vrad0 = k.vradmed[i];
    dens0 = k.sigmamed[i];
    energ0 = k.energymed[i];
  }
  const int zero_here = k.zero_vrad &&
      (((k.rmed[i] < k.wkzrmin) && (i == 0 || i == 1)) || ((k.rmed[i] > k.wkzrmax) && (i == nr - 1)));
  // one divisor per ring: each quotient is the correctly rounded x / (1 +
  // lambda) through its reciprocal; a batch's loads are all in flight
  // before its first store
  const double den = 1.0 + lambda, rden = 1.0 / den;
  for (int j0 = threadIdx.x; j0 < ns; j0 += RING_U * FB_BS) {
    double vr[RING_U], vt[RING_U], rh[RING_U], en[RING_U];
#pragma unroll
    for (int u = 0; u < RING_U; u++) {
      const int j = j0 + u * FB_BS;
      if (j < ns) {
        vr[u] = k.vr[base + j];
        vt[u] = k.vt[base + j];
        rh[u] = k.rho[base + j];
        en[u] = k.energy ? k.e[base + j] : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < RING_U; u++) {
      const int j = j0 + u * FB_BS;
      if (j >= ns) continue;
      const size_t l = base + j;
      if (zero_here) {
        k.vr[l] = 0.0;
        k.rho[l] = dens0;
        k.vt[l] = vtheta0;
      } else {
        k.vr[l] = fb_quot(vr[u] + lambda * vrad0, den, rden);
        k.vt[l] = fb_quot(vt[u] + lambda * vtheta0, den, rden);
        k.rho[l] = fb_quot(rh[u] + lambda * dens0, den, rden);
      }
      if (k.energy) k.e[l] = fb_quot(en[u] + lambda * energ0, den, rden);
    }
  }
}

void fb_launch_damping(const KP &k, double dt_override, cudaStream_t s)
{
  if (k.n_damp_rings > 0) fb_launch(k_damping, k.n_damp_rings, FB_BS, 0, s, k, dt_override);
}

// ------------------------------------------------------------ diagnostics
// GasTotalMass (SideEuler.c:15-40) and GasMomentum (SideEuler.c:114-147)
__global__ void __launch_bounds__(FB_BS) k_diag(KP k, double *out)
{
  fb_grid_dependency();
  __shared__ double sh[32];
  const int ns = k.ns;
  const size_t n = (size_t)k.nr * ns;
  double m = 0.0, p = 0.0;
  for (size_t l = (size_t)blockIdx.x * FB_BS + threadIdx.x; l < n; l += (size_t)gridDim.x * FB_BS) {
    const int i = (int)(l / ns), j = (int)(l - (size_t)i * ns);
    m += k.surf[i] * k.rho[l];
    double vt_cent;
    if (j < ns - 1)
      vt_cent = 0.5 * (k.vt[l] + k.vt[l + 1]) + k.rmed[i] * omf(k);
    else
      vt_cent = 0.5 * (k.vt[l] + k.vt[(size_t)i * ns]) + k.rmed[i] * omf(k);
    p += k.surf[i] * k.rho[l] * k.rmed[i] * vt_cent;
  }
  m = block_sum<FB_BS>(m, sh);
  p = block_sum<FB_BS>(p, sh);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = m;
    out[2 * blockIdx.x + 1] = p;
  }
}

void fb_launch_diag(const KP &k, double *out2, cudaStream_t s)
{
  fb_launch(k_diag, k.n_partial_blocks, FB_BS, 0, s, k, out2);
}

// Derived output fields (layout (nr+1)*ns; ring nr zero)
__global__ void __launch_bounds__(FB_BS) k_derived(KP k, int which, double *out)
{
  fb_grid_dependency();
  const int ns = k.ns;
  const size_t n = (size_t)k.nr * ns;
  for (size_t l = (size_t)blockIdx.x * FB_BS + threadIdx.x; l < n; l += (size_t)gridDim.x * FB_BS) {
    double v = 0.0;
    switch (which) {
      case 0:  // ComputeTemperatureField (SourceEuler.c:2440-2460)
        v = k.energy ? 1.0 / 1.0 * (k.gamma - 1.0) * k.e[l] / k.rho[l] : 1.0 / 1.0 * k.pres[l] / k.rho[l];
        break;
      case 1: v = k.pot[l]; break;
      case 2: v = k.pres[l]; break;
      case 3: v = k.cs[l]; break;
      case 4: v = k.divv[l]; break;
      case 5: v = k.vischeat[l]; break;
      case 6: v = k.sg_accr[l]; break;
      case 7: v = k.sg_acct[l]; break;
      default: v = 0.0;
    }
    out[l] = v;
  }
}

void fb_launch_derived(const KP &k, int which, double *out, cudaStream_t s)
{
  const size_t n = (size_t)k.nr * k.ns;
  fb_launch(k_derived, (int)((n + FB_BS - 1) / FB_BS), FB_BS, 0, s, k, which, out);
}

// Start of one AlgoGas call: dtemp = 0 (SourceEuler.c:333) and the loop flags.
__global__ void k_begin_dt(KP k, double DT)
{
  fb_grid_dependency();
  fb_ctl *c = k.ctl;
  c->DT = DT;
  c->dtemp = 0.0;
  c->done = 0;
  c->substeps = 0;
  c->status = 0;
  c->nonfinite = 0;
  c->crash_substeps = 0;
  c->neg_dens_substeps = 0;
}

void fb_launch_begin_dt(const KP &k, double DT, cudaStream_t s) { fb_launch(k_begin_dt, 1, 1, 0, s, k, DT); }

// Lets a kernel take all the dynamic shared memory the device offers beside
// its static part.  The limit is a per-function attribute shared by every
// context in the process, so it is raised once to the device maximum rather
// than set to one grid's need (contexts of different sizes coexist).
int fb_allow_max_dynamic_smem(const void *func)
{
  int dev = 0, maxopt = 0;
  cudaFuncAttributes fa;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, func) != cudaSuccess)
    return FB_ERR_CUDA;
  const int dyn = maxopt - (int)fa.sharedSizeBytes;
  return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) == cudaSuccess ? FB_OK
                                                                                                    : FB_ERR_CUDA;
}

int fb_gas_prepare(int ns, int energy)
{
  const int NQ = energy ? 6 : 5;
  const size_t smem = (size_t)FB_AZI_RINGS(NQ) * ns * sizeof(double);
  int dev = 0, maxopt = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem + 32 * sizeof(double) > (size_t)maxopt) return FB_ERR_UNSUPPORTED;
  if (fb_azi_E_auto(ns) > 4 || ns < 16) return FB_ERR_UNSUPPORTED;
#define AZI_FNS(NQ, F, WD)                                                                               \
  (const void *)k_transport_azimuthal<NQ, 1, F, WD>, (const void *)k_transport_azimuthal<NQ, 2, F, WD>,  \
      (const void *)k_transport_azimuthal<NQ, 3, F, WD>, (const void *)k_transport_azimuthal<NQ, 4, F, WD>
#define AZP_FNS(NQ, F)                                                                                   \
  (const void *)k_transport_azimuthal_packed<NQ, 1, F>, (const void *)k_transport_azimuthal_packed<NQ, 2, F>, \
      (const void *)k_transport_azimuthal_packed<NQ, 3, F>, (const void *)k_transport_azimuthal_packed<NQ, 4, F>
  const void *fns[] = {AZI_FNS(5, false, false), AZI_FNS(5, true, false), AZI_FNS(6, false, false),
                       AZI_FNS(6, true, false),  AZI_FNS(5, false, true),  AZI_FNS(5, true, true),
                       AZI_FNS(6, false, true),  AZI_FNS(6, true, true),   AZP_FNS(5, false),
                       AZP_FNS(5, true),         AZP_FNS(6, false),        AZP_FNS(6, true)};
#undef AZI_FNS
#undef AZP_FNS
  {
    int rc = fb_allow_max_dynamic_smem((const void *)k_cfl);  // 3 nsec doubles of cell values
    if (rc) return rc;
  }
#define AZS_FNS(NQ, EE)                                                                  \
  (const void *)k_transport_azimuthal_staged<NQ, EE, 256>,                               \
      (const void *)k_transport_azimuthal_staged<NQ, EE, 384>,                           \
      (const void *)k_transport_azimuthal_staged<NQ, EE, 512>,                           \
      (const void *)k_transport_azimuthal_staged<NQ, EE, 768>
  {
    const void *sfns[] = {AZS_FNS(5, 2), AZS_FNS(5, 3), AZS_FNS(5, 4), AZS_FNS(6, 2), AZS_FNS(6, 3), AZS_FNS(6, 4)};
    for (const void *f : sfns) {
      int rc = fb_allow_max_dynamic_smem(f);
      if (rc) return rc;
    }
  }
#undef AZS_FNS
  for (const void *f : fns) {
    int rc = fb_allow_max_dynamic_smem(f);
    if (rc) return rc;
    // the whole unified L1 as shared memory: two rings' CTAs per SM where they fit
    if (cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess)
      return FB_ERR_CUDA;
  }
  return FB_OK;
}

// Loop condition of the captured substep graph: keep going while the
// controller has not reached DT (SourceEuler.c:398) and nothing failed; the
// cap bounds the loop even if the time step collapses.
__global__ void k_loop_cond(KP k, cudaGraphConditionalHandle h, int cap)
{
  fb_grid_dependency();
  fb_ctl *c = k.ctl;
  int go = (!c->done && !c->status) ? 1 : 0;
  if (go && c->substeps >= cap) {
    c->status = FB_ERR_SUBSTEPS;
    go = 0;
  }
  cudaGraphSetConditional(h, go);
}

void fb_launch_loop_cond(const KP &k, cudaGraphConditionalHandle h, int cap, cudaStream_t s)
{
  fb_launch(k_loop_cond, 1, 1, 0, s, k, h, cap);
}
