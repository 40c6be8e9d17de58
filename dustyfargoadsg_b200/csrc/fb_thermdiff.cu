// fb_thermdiff.cu -- thermal diffusion of the energy equation: SubStep0
// (src/SourceEuler.c:722-762) with ComputeEntropyDiffusion (:1740-1789),
// ComputeRadiativeDiffusion (:1791-1876) and the implicit solver
// SORsolver_RadiativeDiffusion (:1878-2052).
//
// Per substep, after the controller has set dt and before the sound speed:
//  1. k_td_fields: per cell the entropy logarithm log((gamma-1) e /
//     Sigma^gamma) (0 where the argument is not positive) and the
//     temperature (gamma-1) e / Sigma;
//  2. explicit radiative diffusion: k_td_coefficient, the flux-limited (Kley
//     1989) diffusion coefficient K per cell of rings 0..nr-2 (ring nr-1
//     reads ring nr-2's, as the reference copies it), from the opacity of
//     the current state;
//  3. k_td_apply: the entropy and radiative sources of rings 1..nr-2 and
//     the explicit update energy += EntropyDiff dt, then += RadiativeDiff dt
//     (two roundings, as the reference adds them one after the other);
//  4. implicit radiative diffusion: the opacity of the (explicitly updated)
//     state, k_td_fields again for the temperature, k_td_coefficient (chi per
//     cell), k_sor_coef (the coefficients a..f of rings 1..nr-2 and each CTA's part
//     of the initial residual norm), then k_sor_solve.
//
// k_sor_solve is one persistent kernel of as many CTAs as the GPU holds at
// once.  An iteration is the reference's two chessboard passes: pass 1
// updates the cells (i, j) of rings 1..nr-2 with i + j odd, pass 2 those
// with i + j even.  A cell's five-point stencil reaches only cells of the
// other colour (with an even NSEC the azimuthal wrap keeps that true), so
// the cells of one pass are independent and updating them in parallel gives
// exactly the reference's sequential sweep.  Between the passes and after
// the second the CTAs meet at a grid barrier (an atomic arrival counter and
// a generation word; every wait is bounded: one that runs out sets
// FB_ERR_TIMEOUT in the control block and the kernel returns).  The
// residual norm sum(|resid|) of an iteration is summed per CTA and the
// partial sums, double-buffered by iteration parity, are added by every CTA
// in the same fixed order, so every CTA takes the same convergence decision
// (norm < epsilonSOR x initial norm).  The norm's order of summation differs
// from the reference's sequential one by rounding only, which can move the
// decision only for a norm within ~1e-16 relative of the threshold.
// On convergence Energy = Sigma T / (gamma-1) on rings 0..nr-1; after
// MAXITS iterations without it the energy is left as it was, as the
// reference leaves it.  omegaSOR and niterbuf then evolve as SubStep0 has
// them evolve.
#include <math.h>
#include "fb_dev.cuh"

#define TD_BS 256

// ---------------------------------------------------------------- fields
// entropy logarithm (ComputeEntropyDiffusion's TempInt) and temperature
// (ComputeRadiativeDiffusion's and the solver's TempInt), rings 0..nr-1
__global__ void __launch_bounds__(TD_BS) k_td_fields(KP k, int want_s, int want_t)
{
  fb_grid_dependency();
  const size_t n = (size_t)k.nr * k.ns;
  for (size_t l = (size_t)blockIdx.x * TD_BS + threadIdx.x; l < n; l += (size_t)gridDim.x * TD_BS) {
    const double energy = k.e[l], dens = k.rho[l];
    if (want_s) {
      const double buf = (k.gamma - 1.0) * energy / pow(dens, k.gamma);
      double s = 0.0;
      if (buf > 0.0) s = log(buf);
      k.td_s[l] = s;
    }
    if (want_t) k.td_t[l] = (k.gamma - 1.0) * energy / dens;
  }
}

// Flux limiter lambda(R) of Kley (1989) as the reference writes it
static __device__ __forceinline__ double td_lambda(double Rl)
{
  if (Rl <= 2.0) return 2. / (3. + sqrt(9.0 + 10.0 * Rl * Rl));
  return 10. / (10. * Rl + 9.0 + sqrt(180. * Rl + 81.));
}

// R of the flux limiter at cell (i, j) of the temperature field t
static __device__ __forceinline__ double td_rl(const KP &k, const double *t, int i, int j, size_t l)
{
  const int ns = k.ns;
  const size_t lip = l + ns, ljp = (j == ns - 1) ? (size_t)i * ns : l + 1;
  const double a = k.invdiffrmed[i + 1] * (t[lip] - t[l]);
  const double b = k.invrmed[i] * k.invdphi * (t[ljp] - t[l]);
  const double gradT = sqrt(a * a + b * b);
  return (8.0 * sqrt(k.gamma * t[l]) * k.p15[i] / k.rho[l] / k.opacity[l]) * (gradT / t[l]);
}

// K (explicit, :1826-1838) or chi (implicit, :1921-1933) of rings 0..nr-2
__global__ void __launch_bounds__(TD_BS) k_td_coefficient(KP k, int implicit)
{
  fb_grid_dependency();
  const int ns = k.ns;
  const size_t n = (size_t)(k.nr - 1) * ns;
  for (size_t l = (size_t)blockIdx.x * TD_BS + threadIdx.x; l < n; l += (size_t)gridDim.x * TD_BS) {
    const int i = (int)(l / ns), j = (int)(l - (size_t)i * ns);
    const double *t = k.td_t;
    const double lambda = td_lambda(td_rl(k, t, i, j, l));
    const double dens = k.rho[l], opacity = k.opacity[l];
    if (!implicit)
      k.td_k[l] = 32.0 * k.sigma_sb * lambda * sqrt(k.gamma) * pow(t[l], 3.5) * k.p15[i] / dens / opacity;
    else
      k.td_k[l] = 64.0 * k.sigma_sb * lambda * k.gamma * (k.gamma - 1.0) * pow(t[l], 4.0) * pow(k.rmed[i], 3.0) *
                  pow(dens, -2.0) / opacity;
  }
}

// the coefficient at cell l of ring i, ring nr-1 reading ring nr-2's
static __device__ __forceinline__ double td_coef(const KP &k, int i, size_t l)
{
  return (i == k.nr - 1) ? k.td_k[l - k.ns] : k.td_k[l];
}

// Explicit thermal diffusion: EntropyDiff (:1770-1788) and RadiativeDiff
// (:1845-1874) of rings 1..nr-2 (the other rings' sources stay zero, as the
// reference never writes them), then SubStep0's update of rings 0..nr-1
// (:737-746).  Each cell reads only the entropy and temperature fields and
// K, none of which this kernel writes, so the update is made in place.
__global__ void __launch_bounds__(TD_BS) k_td_apply(KP k)
{
  fb_grid_dependency();
  const int ns = k.ns, nr = k.nr;
  const double dt = k.ctl->dt;
  const size_t n = (size_t)nr * ns;
  for (size_t l = (size_t)blockIdx.x * TD_BS + threadIdx.x; l < n; l += (size_t)gridDim.x * TD_BS) {
    const int i = (int)(l / ns), j = (int)(l - (size_t)i * ns);
    double energy = k.e[l];
    if (i >= 1 && i <= nr - 2) {
      const size_t lip = l + ns, lim = l - ns;
      const size_t ljp = (j == ns - 1) ? (size_t)i * ns : l + 1;
      const size_t ljm = (j == 0) ? (size_t)i * ns + ns - 1 : l - 1;
      const double irm = k.invrmed[i];
      if (k.ent_diff) {
        const double *t = k.td_s;
        const double laplacien =
            k.invdiffrsup[i] * irm *
                (k.rsup[i] * k.invdiffrmed[i + 1] * (t[lip] - t[l]) - k.rinf[i] * k.invdiffrmed[i] * (t[l] - t[lim])) +
            irm * irm * k.invdphi * k.invdphi * (t[ljp] + t[ljm] - 2.0 * t[l]);
        const double ed = energy * k.diffusivity * laplacien;
        k.td_ent[l] = ed;
        energy += ed * dt;
      }
      if (k.rad_diff == 1) {
        const double *t = k.td_t;
        const double kl = k.td_k[l], kip = td_coef(k, i + 1, lip), kim = k.td_k[lim];
        const double kjp = k.td_k[ljp], kjm = k.td_k[ljm];
        const double rm = k.rmed[i], rmp = k.rmed[i + 1], rmm = k.rmed[i - 1];
        const double KRsup = ((rmp - k.rsup[i]) * kl + (k.rsup[i] - rm) * kip) / (rmp - rm);
        const double KRinf = ((rm - k.rinf[i]) * kim + (k.rinf[i] - rmm) * kl) / (rm - rmm);
        const double KPhisup = 0.5 * (kl + kjp);
        const double KPhiinf = 0.5 * (kl + kjm);
        const double divF =
            k.invdiffrsup[i] * irm *
                (k.rsup[i] * KRsup * k.invdiffrmed[i + 1] * (t[lip] - t[l]) -
                 k.rinf[i] * KRinf * k.invdiffrmed[i] * (t[l] - t[lim])) +
            irm * irm * k.invdphi * k.invdphi * (KPhisup * (t[ljp] - t[l]) - KPhiinf * (t[l] - t[ljm]));
        const double rd = 2.0 * sqrt(k.gamma * t[l]) * k.p15[i] * divF;
        k.td_rad[l] = rd;
        energy += rd * dt;
      }
    }
    k.e[l] = energy;
  }
}

// ------------------------------------------------------------------ solver
// Sum over the CTA in a fixed order (warp trees, then the warps' sums)
static __device__ double td_block_sum(double v, double *sh)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[0] = v;
  }
  __syncthreads();
  const double r = sh[0];
  __syncthreads();
  return r;
}

// Sum of the n partial sums p[0..n) in a fixed order (every CTA that calls
// it gets the same value); the partials come from other CTAs: read past L1
static __device__ double td_partials_sum(const double *p, int n, double *sh)
{
  double v = 0.0;
  for (int q = threadIdx.x; q < n; q += blockDim.x) v += __ldcg(p + q);
  return td_block_sum(v, sh);
}

// the five-point residual of the solver's equation at cell l
// (SourceEuler.c:1993, 2012) with the temperatures read past L1
static __device__ __forceinline__ double sor_resid(const KP &k, const double *t, int i, int j, size_t l)
{
  const int ns = k.ns;
  const size_t lip = l + ns, lim = l - ns;
  const size_t ljp = (j == ns - 1) ? (size_t)i * ns : l + 1;
  const size_t ljm = (j == 0) ? (size_t)i * ns + ns - 1 : l - 1;
  return k.sor_c[0][l] * __ldcg(t + lip) + k.sor_c[1][l] * __ldcg(t + lim) + k.sor_c[2][l] * __ldcg(t + ljp) +
         k.sor_c[3][l] * __ldcg(t + ljm) + k.sor_c[4][l] * __ldcg(t + l) - k.sor_c[5][l];
}

// The coefficients a..f of the cells of rings 1..nr-2 (SourceEuler.c:
// 1941-1966) from chi and the temperature, and this CTA's part of the
// initial residual norm (:1977-1991), stored at sor_part[2 G + CTA].  The
// CTA resets the solver's barrier counter first (no barrier is active now).
__global__ void __launch_bounds__(TD_BS) k_sor_coef(KP k)
{
  fb_grid_dependency();
  __shared__ double sh[32];
  const int ns = k.ns, nr = k.nr, G = gridDim.x;
  if (blockIdx.x == 0 && threadIdx.x == 0) k.sor_bar[0] = 0u;
  const double dt = k.ctl->dt;
  const double *chi = k.td_k, *t = k.td_t;
  const size_t n0 = (size_t)ns, n1 = (size_t)(nr - 1) * ns;
  double acc = 0.0;
  for (size_t l = n0 + (size_t)blockIdx.x * TD_BS + threadIdx.x; l < n1; l += (size_t)G * TD_BS) {
    const int i = (int)(l / ns), j = (int)(l - (size_t)i * ns);
    const size_t lip = l + ns, lim = l - ns;
    const size_t ljp = (j == ns - 1) ? (size_t)i * ns : l + 1;
    const size_t ljm = (j == 0) ? (size_t)i * ns + ns - 1 : l - 1;
    const double cl = chi[l], cip = td_coef(k, i + 1, lip), cim = chi[lim];
    const double rm = k.rmed[i], rmp = k.rmed[i + 1], rmm = k.rmed[i - 1];
    const double chiRsup = ((rmp - k.rsup[i]) * cl + (k.rsup[i] - rm) * cip) / (rmp - rm);
    const double chiRinf = ((rm - k.rinf[i]) * cim + (k.rinf[i] - rmm) * cl) / (rm - rmm);
    const double chiPhisup = 0.5 * (cl + chi[ljp]);
    const double chiPhiinf = 0.5 * (cl + chi[ljm]);
    const double irm = k.invrmed[i];
    const double a = -dt * k.rsup[i] * k.invdiffrsup[i] * chiRsup * irm * k.invdiffrmed[i + 1];
    const double b = -dt * k.rinf[i] * k.invdiffrsup[i] * chiRinf * irm * k.invdiffrmed[i];
    const double c = -dt * chiPhisup * irm * irm * k.invdphi * k.invdphi;
    const double d = -dt * chiPhiinf * irm * irm * k.invdphi * k.invdphi;
    const double e = 1.0 - a - b - c - d;
    const double f = t[l];
    k.sor_c[0][l] = a;
    k.sor_c[1][l] = b;
    k.sor_c[2][l] = c;
    k.sor_c[3][l] = d;
    k.sor_c[4][l] = e;
    k.sor_c[5][l] = f;
    const double resid = a * t[lip] + b * t[lim] + c * t[ljp] + d * t[ljm] + e * t[l] - f;
    acc += fabs(resid);
  }
  acc = td_block_sum(acc, sh);
  if (threadIdx.x == 0) k.sor_part[2 * G + blockIdx.x] = acc;
}

#define SOR_WAIT_LIMIT (1 << 24)  // polls of the generation word (~1.6 s with the back-off)

// Grid barrier of the solver's CTAs: the last to arrive resets the counter
// and advances the generation; the others wait for the generation to move,
// a bounded number of polls.  Returns false (for the whole CTA) if the wait
// ran out.
static __device__ bool sor_barrier(unsigned int *bar, unsigned int &gen, int *flag)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    if (atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicAdd(&bar[1], 1u);
    } else {
      long long it = 0;
      while (atomicAdd(&bar[1], 0u) == gen) {
        if (++it > SOR_WAIT_LIMIT) { ok = 0; break; }
        __nanosleep(100);
      }
    }
    __threadfence();
    *flag = ok;
  }
  __syncthreads();
  gen += 1u;
  return *flag != 0;
}

__global__ void __launch_bounds__(TD_BS) k_sor_solve(KP k)
{
  __shared__ double sh[32];
  __shared__ int flag;
  const int ns = k.ns, nr = k.nr, G = gridDim.x, half = ns / 2;
  __shared__ unsigned int g0;  // the barrier's generation at the start
  if (threadIdx.x == 0) g0 = atomicAdd(&k.sor_bar[1], 0u);
  __syncthreads();
  unsigned int gen = g0;
  const double omega = k.ctl->sor_omega;
  const double init = td_partials_sum(k.sor_part + 2 * G, G, sh);
  double *t = k.td_t;
  const size_t ncol = (size_t)(nr - 2) * half;
  int n, converged = 0;
  for (n = 1; n <= FB_SOR_MAXITS; n++) {
    double acc = 0.0;
    for (int pass = 0; pass < 2; pass++) {
      // pass 1: the cells with i + j odd (jchess starts at 0 on ring 1),
      // pass 2: i + j even
      for (size_t c = (size_t)blockIdx.x * TD_BS + threadIdx.x; c < ncol; c += (size_t)G * TD_BS) {
        const int i = 1 + (int)(c / half), jj = (int)(c - (size_t)(i - 1) * half);
        const int j = 2 * jj + (pass == 0 ? ((i - 1) & 1) : (i & 1));
        const size_t l = (size_t)i * ns + j;
        const double resid = sor_resid(k, t, i, j, l);
        acc += fabs(resid);
        __stcg(t + l, __ldcg(t + l) - omega * resid / k.sor_c[4][l]);
      }
      if (pass == 0 && !sor_barrier(k.sor_bar, gen, &flag)) goto timeout;
    }
    acc = td_block_sum(acc, sh);
    if (threadIdx.x == 0) k.sor_part[(n & 1) * G + blockIdx.x] = acc;
    if (!sor_barrier(k.sor_bar, gen, &flag)) goto timeout;
    if (td_partials_sum(k.sor_part + (n & 1) * G, G, sh) < FB_SOR_EPS * init) {
      converged = 1;
      break;
    }
  }
  if (converged) {  // Energy from the solved temperature (:2031-2036)
    const size_t nc = (size_t)nr * ns;
    for (size_t l = (size_t)blockIdx.x * TD_BS + threadIdx.x; l < nc; l += (size_t)G * TD_BS)
      k.e[l] = k.rho[l] * __ldcg(t + l) / (k.gamma - 1.0);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {  // SubStep0's omegaSOR and niterbuf (:751-759)
    fb_ctl *c = k.ctl;
    const int niter = n;  // MAXITS + 1 when the solve did not converge
    const double best = c->sor_omega;
    double w = c->sor_omega;
    if (!(niter < c->sor_niterbuf)) {
      w *= 0.9999;
      if ((w >= 2.0) || (w <= 1.0)) w = best;
    }
    c->sor_omega = w;
    c->sor_niterbuf = niter;
    c->sor_iters = niter;
  }
  return;
timeout:
  if (threadIdx.x == 0) {
    k.ctl->status = FB_ERR_TIMEOUT;
    k.ctl->done = 1;
  }
}

// ------------------------------------------------------------------ launch
static int td_grid(const KP &k)
{
  const size_t n = (size_t)k.nr * k.ns;
  const size_t g = (n + TD_BS - 1) / TD_BS;
  return (int)(g < 4096 ? g : 4096);
}

// CTAs of the solver: at most two per SM and no more than the SM holds, so
// that all of them are resident together (the launch is cooperative too)
int fb_sor_grid(void)
{
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sor_solve, TD_BS, 0) != cudaSuccess || per < 1) {
    cudaGetLastError();
    return 0;
  }
  return sms * (per < 2 ? per : 2);
}

int fb_launch_substep0(const KP &k, cudaStream_t s)
{
  int n = 0;
  const int g = td_grid(k);
  if (k.ent_diff || k.rad_diff == 1) {  // explicit sources and update (:737-746)
    fb_launch(k_td_fields, g, TD_BS, 0, s, k, k.ent_diff, k.rad_diff == 1 ? 1 : 0);
    n++;
    if (k.rad_diff == 1) {  // the opacity of this state was computed before the CFL kernel
      fb_launch(k_td_coefficient, g, TD_BS, 0, s, k, 0);
      n++;
    }
    fb_launch(k_td_apply, g, TD_BS, 0, s, k);
    n++;
  }
  if (k.rad_diff == 2) {  // implicit radiative diffusion (:749-760)
    n += fb_launch_opacity_now(k, s);
    fb_launch(k_td_fields, g, TD_BS, 0, s, k, 0, 1);
    fb_launch(k_td_coefficient, g, TD_BS, 0, s, k, 1);
    fb_launch(k_sor_coef, k.sor_grid, TD_BS, 0, s, k);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(k.sor_grid);
    cfg.blockDim = dim3(TD_BS);
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_sor_solve, k);
    n += 4;
  }
  return n;
}

// The explicit radiative diffusion's time-step limit invdt6 of every cell
// of rings 1..nr-1 (SourceEuler.c:1413-1424), into the RadiativeDiff
// scratch field (free until SubStep0) for the CFL kernel that follows.  The
// Temperature field of the reference is (gamma-1) e / Sigma of the current
// state on rings 0..nr-1 and zero on ring nr, which it never writes; the
// opacity is the one computed for this state just before.
__global__ void __launch_bounds__(TD_BS) k_td_cfl(KP k)
{
  fb_grid_dependency();
  const int ns = k.ns, nr = k.nr;
  const size_t n0 = (size_t)ns, n1 = (size_t)nr * ns;
  for (size_t l = n0 + (size_t)blockIdx.x * TD_BS + threadIdx.x; l < n1; l += (size_t)gridDim.x * TD_BS) {
    const int i = (int)(l / ns), j = (int)(l - (size_t)i * ns);
    const size_t ljp = (j == ns - 1) ? (size_t)i * ns : l + 1;
    const double dens = k.rho[l];
    const double T = (k.gamma - 1.0) * k.e[l] / dens;
    const double Tip = (i + 1 <= nr - 1) ? (k.gamma - 1.0) * k.e[l + ns] / k.rho[l + ns] : 0.0;
    const double Tjp = (k.gamma - 1.0) * k.e[ljp] / k.rho[ljp];
    const double opacity = k.opacity[l];
    const double a = k.invdiffrmed[i + 1] * (Tip - T), b = k.invrmed[i] * k.invdphi * (Tjp - T);
    const double gradT = sqrt(a * a + b * b);
    const double Rl = (8.0 * sqrt(k.gamma * T) * k.p15[i] / dens / opacity) * gradT / T;
    const double lambda = td_lambda(Rl);
    const double chicoeff = 64.0 * lambda * k.sigma_sb * k.gamma * (k.gamma - 1.0) * pow(T, 4.0) / opacity /
                            (dens * dens) * pow(k.rmed[i], 3.0);
    k.td_rad[l] = chicoeff * 4.0 / k.mindx2[i];
  }
}

int fb_launch_td_cfl(const KP &k, cudaStream_t s)
{
  fb_launch(k_td_cfl, td_grid(k), TD_BS, 0, s, k);
  return 1;
}
