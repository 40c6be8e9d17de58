// fb_dust.cu -- Lagrangian dust particles of AlgoGas (src/SourceEuler.c:504-531)
// on the GPU: SemiUpdateDustPositions (src/DustUpdate.c:6-265), the TSC
// interpolation of the gas onto the particles (src/Dsys.c:265-1149) and
// UpdateDustVelocities (src/DustUpdate.c:267-435).  FP64, one thread per
// particle, particles kept as a structure of arrays in the reference's index
// order.  The gas grids are read through L2 (a 256x768 ring set is 1.5 MB a
// field), so the per-particle stencil gathers are L2 hits.
//
// Turbulent kicks and their random stream.  The reference draws the kicks
// in particle order from the one drand48 stream through two Gaussian
// generators (myrandn_rad, myrandn_phi, src/DustUpdate.c:438-485), each a
// Marsaglia polar method that hands out the second deviate of its pair on
// its next call.  Both are called once per kicked particle, so kick number m
// (counted over the whole run) takes its radial deviate from accepted pair
// 2*(m/2) and its azimuthal one from accepted pair 2*(m/2)+1 -- x1 for even
// m, x2 for odd m -- where "accepted pairs" are the Marsaglia acceptances
// among consecutive uniform pairs of the stream.  The GPU reproduces that
// stream exactly: a scan ranks the kicked particles, candidate uniform pairs
// are drawn in parallel with the LCG's closed-form skip-ahead
// (X_{n+m} = a^m X_n + c (a^m - 1)/(a - 1) mod 2^48, evaluated by binary
// powering), the accepted candidates are compacted in stream order, and the
// stream position is advanced past the last candidate used.
#include <cuda_runtime.h>
#include <math.h>
#include "fb_dev.cuh"

#define D_BS 256
#define SCAN_BS 1024

static const unsigned long long LCG_A = 0x5DEECE66Dull, LCG_C = 0xBull, M48 = 0xFFFFFFFFFFFFull;

// The recurrence applied 2^i times is again affine, X <- (A_i X + C_i) mod
// 2^48, with A_0 = a, C_0 = c, A_{i+1} = A_i^2, C_{i+1} = (A_i + 1) C_i.
struct LcgJumps {
  unsigned long long A[48], C[48];
  constexpr LcgJumps() : A(), C()
  {
    unsigned long long a = LCG_A, c = LCG_C;
    for (int i = 0; i < 48; i++) {
      A[i] = a;
      C[i] = c;
      c = ((a + 1) * c) & M48;
      a = (a * a) & M48;
    }
  }
};
__constant__ LcgJumps c_jumps = LcgJumps();

// X_{n+m} from X_n: one affine map per set bit of m (the maps commute).  The
// loop runs over the bit positions, so a warp whose threads skip by similar
// m reads the same table entry in each iteration.
static __device__ __forceinline__ unsigned long long lcg_skip(unsigned long long x, unsigned long long m)
{
  for (int i = 0; m; i++, m >>= 1)
    if (m & 1ull) x = (c_jumps.A[i] * x + c_jumps.C[i]) & M48;
  return x;
}

// drand48's value of a state: X / 2^48, exact in double
static __device__ __forceinline__ double u48(unsigned long long x) { return (double)x * 0x1p-48; }

static __device__ __forceinline__ double wrap_azimuth(const PP &pp, double th)
{
  // src/DustUpdate.c:44-47 and 130-133
  if (th < pp.aziinf0) th += (pp.azisupl - pp.aziinf0);
  if (th > pp.azisupl) th -= (pp.azisupl - pp.aziinf0);
  return th;
}

// TSC weight of one axis (src/Dsys.c:451-463)
// The reference's pow(x, 1.5), pow(x, -2.0) and pow(x, -3.0) (x > 0) as a
// square root, products and one reciprocal: within a few ulp of the exact
// power, as the library pow is, at a small part of its cost.
static __device__ __forceinline__ double pow15(double x) { return x * sqrt(x); }
static __device__ __forceinline__ double powm2(double x) { return 1.0 / (x * x); }
static __device__ __forceinline__ double powm3(double x) { return 1.0 / (x * x * x); }

// The triangular-shaped-cloud weight at distance d for a cell of width
// delta; rdelta = 1/delta rounded, so that each quotient by delta is the
// correctly rounded one through fb_quot (no division).
static __device__ __forceinline__ double tsc_weight(double d, double delta, double rdelta)
{
  double w = 0.0;
  if (d < 0.5 * delta) w = 0.75 - fb_quot(fb_quot(d * d, delta, rdelta), delta, rdelta);
  if ((d >= 0.5 * delta) && (d <= 1.5 * delta)) {
    const double q = fb_quot(d, delta, rdelta);
    w = 0.5 * (1.5 - q) * (1.5 - q);
  }
  if (d > 1.5 * delta) w = 0.0;
  return w;
}

// The reference finds rings by linear searches over the radii (Dsys.c:364,
// DustUpdate.c:73, Viscosity.c:31).  The same indices come from a first
// guess by the grid law and a correction against the sorted radii.
static __device__ __forceinline__ int ring_guess(const PP &pp, double x, int n)
{
  const double u = pp.log_grid ? log(x * pp.ring_inv_r0) * pp.ring_inv_step : (x - pp.ring_r0) * pp.ring_inv_step;
  return (u > 0.0) ? (int)fmin(u, (double)(n - 1)) : 0;
}
// largest index g in [0, n) with a[g] <= x, given a[0] <= x (the linear
// search `while (x >= a[i] && i <= n-1) i++; i--`)
static __device__ __forceinline__ int last_not_above(const PP &pp, const double *a, int n, double x)
{
  int g = ring_guess(pp, x, n);
  while (g > 0 && a[g] > x) g--;
  while (g < n - 1 && a[g + 1] <= x) g++;
  return g;
}
// first index in [0, n - 1) with a[idx] >= x, else n - 1 (the search
// `while (a[i] < x) i++` stopped at the last entry)
static __device__ __forceinline__ int first_not_below_clamped(const PP &pp, const double *a, int n, double x)
{
  int g = ring_guess(pp, x, n);
  while (g > 0 && a[g - 1] >= x) g--;
  while (g < n - 1 && a[g] < x) g++;
  return g;
}

// FViscosity (src/Viscosity.c:23-69) at a particle radius.  The reference's
// search `while (GlobalRmed[i] < rad) i++` has no upper bound and runs past
// the last ring for radii beyond Rmed[nr-1]; here it stops at the last ring.
static __device__ double viscosity_at(const KP &k, const PP &pp, double rad)
{
  if (k.visc_mode == 1) {
    const int i = first_not_below_clamped(pp, k.rmed, k.nr, rad);  // <= nr-1
    return k.alpha * k.gcs[i] * k.gcs[i] * pow15(rad);
  }
  return (k.visc_mode == 2) ? k.nu_const : 0.0;
}

// Stokes number with the Paardekooper (2007) drag law (src/Dsys.c:724-764).
// pow(x,2.0) and pow(x,-1.0) are written as the product and the reciprocal
// the reference's compiler turns them into.  AspectRatio(rp) is ASPECTRATIO
// for the supported parameter set (TRANSITIONRATIO = 1, LAMBDADOUBLING = 0).
static __device__ double stokes_number(const PP &pp, double size, double rp, double vrp, double vtp,
                                       double vrg, double vtg, double csg, double densg)
{
  const double densg_cgs = 0.1 * densg * pp.unit_mass * pp.inv_unit_length2;
  const double lambda = 3.34e-8 * (1.0 / densg_cgs) * pp.aspectratio * rp;
  const double Kn = 0.5 * lambda / size;
  const double Mach = sqrt((vrp - vrg) * (vrp - vrg) + (vtp - vtg) * (vtp - vtg)) / csg;
  const double f_D = sqrt(1.0 + 9.0 * M_PI * Mach * Mach / 128.0);
  const double Re = 3.0 * sqrt(FB_PI / 8.0) * Mach / Kn;
  double k_D = 0.0;
  if (Re <= 500.0) {
    k_D = 1.0 + 0.15 * pow(Re, 0.687);
  } else {
    if ((Re > 500.0) && (Re <= 1500.0)) k_D = 3.96e-6 * pow(Re, 2.4);
    if (Re > 1500.0) k_D = 0.11 * Re;
  }
  const double a3 = 3.0 * Kn + 1.0;
  const double Cdrag = (a3 * a3) * (1.0 / (9.0 * Kn * Kn * f_D + 3.0 * Kn * k_D));
  return 0.5 * M_PI * Cdrag * size * pp.dust_density_cu / densg;
}

// ---------------------------------------------------- 1. drift and flags
// SemiUpdateDustPositions with timestep = 2 dt, drift part (DustUpdate.c:30-56).
// flag = the particle gets a turbulent kick in this substep.
__global__ void __launch_bounds__(D_BS) k_dust_drift(KP k, PP pp)
{
  fb_grid_dependency();
  const int q = blockIdx.x * D_BS + threadIdx.x;
  if (q == 0) pp.dc->min_ts = 1e6;  // reset by every interpolation call (Dsys.c:336)
  if (q >= pp.n) return;
  const double timestep = 2.0 * k.ctl->dt;
  const double rinf0 = k.rinf[0], rsupl = k.rsup[k.nr - 1];
  const double r = pp.r[q];
  int flag = 0;
  if ((r >= rinf0) && (r < rsupl)) {
    const double rn = r + pp.vr[q] * 0.5 * timestep;
    double th = pp.th[q] + pp.vth[q] * r * 0.25 * timestep * (powm2(r) + powm2(rn));
    th = wrap_azimuth(pp, th);
    flag = (pp.feel_turb && (rn >= rinf0) && (rn <= rsupl)) ? 1 : 0;
    if (!flag) th = wrap_azimuth(pp, th);
    pp.r[q] = rn;
    pp.th[q] = th;
  }
  pp.flag[pp.orig[q]] = flag;  // in the reference's order, for the kick ranks
}

// ------------------------------------------------------- 2. scans
static __device__ __forceinline__ int warp_incl_scan(int x)
{
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// exclusive scan of SCAN_BS ints per block; block totals to blocksum
__global__ void __launch_bounds__(SCAN_BS) k_scan_block(const int *in, int *out, int *blocksum, int n)
{
  fb_grid_dependency();
  __shared__ int sh[SCAN_BS / 32];
  const int g = blockIdx.x * SCAN_BS + threadIdx.x;
  const int v = (g < n) ? in[g] : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x = warp_incl_scan(v);
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) sh[lane] = warp_incl_scan(sh[lane]);  // SCAN_BS / 32 == 32 warps
  __syncthreads();
  const int warp_off = (w > 0) ? sh[w - 1] : 0;
  if (g < n) out[g] = warp_off + x - v;
  if (threadIdx.x == SCAN_BS - 1) blocksum[blockIdx.x] = sh[SCAN_BS / 32 - 1];
}

// exclusive scan of nb block sums in place by one CTA of SCAN_BS threads;
// returns the total (valid in every thread)
static __device__ int scan_top(int *blocksum, int nb)
{
  __shared__ int sh[SCAN_BS / 32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < nb; base += SCAN_BS) {
    const int g = base + threadIdx.x;
    const int v = (g < nb) ? blocksum[g] : 0;
    const int x = warp_incl_scan(v);
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) sh[lane] = warp_incl_scan(sh[lane]);
    __syncthreads();
    const int warp_off = (w > 0) ? sh[w - 1] : 0;
    const int c0 = carry;
    if (g < nb) blocksum[g] = c0 + warp_off + x - v;
    __syncthreads();
    if (threadIdx.x == 0) carry = c0 + sh[SCAN_BS / 32 - 1];
    __syncthreads();
  }
  return carry;
}

// Number of kicked particles K of this substep and the accepted pairs it needs.
__global__ void __launch_bounds__(SCAN_BS) k_kick_top(PP pp, int nb)
{
  fb_grid_dependency();
  const int K = scan_top(pp.kick_bsum, nb);
  if (threadIdx.x == 0) {
    fb_dust_ctl *d = pp.dc;
    const long long G = d->kicks;
    d->K = K;
    d->t_start = (G + 1) / 2;  // first pair event not served by the carry
    long long E = 0;
    if (K > 0) {
      E = (G + K - 1) / 2 - d->t_start + 1;
      if (E < 0) E = 0;
    }
    d->npairs = (int)(2 * E);
  }
}

// ------------------------------------------------ 3. Gaussian pairs
// Candidate c takes the uniforms X_{cur+2c+1}, X_{cur+2c+2} of the stream;
// Marsaglia's test of src/DustUpdate.c:449-454 (pow(u,2.0) is u*u).
static __device__ __forceinline__ bool candidate(unsigned long long xcur, long long c, double *u1, double *u2, double *w)
{
  const unsigned long long x1 = lcg_skip(xcur, (unsigned long long)(2 * c + 1));
  const unsigned long long x2 = (LCG_A * x1 + LCG_C) & M48;
  *u1 = 2.0 * u48(x1) - 1.0;
  *u2 = 2.0 * u48(x2) - 1.0;
  *w = (*u1) * (*u1) + (*u2) * (*u2);
  return !(*w >= 1.0 || *w == 0.0);
}

// Candidates examined this substep: enough that the accepted ones (rate pi/4)
// cover npairs with a margin of many standard deviations.
static __device__ __forceinline__ long long candidate_limit(const PP &pp, int npairs)
{
  const long long lim = (long long)npairs * 27 / 20 + 2048;
  return lim < pp.ncand ? lim : pp.ncand;
}

__global__ void __launch_bounds__(D_BS) k_rng_count(PP pp)
{
  fb_grid_dependency();
  __shared__ int sh[D_BS / 32];
  const long long c = (long long)blockIdx.x * D_BS + threadIdx.x;
  const int npairs = pp.dc->npairs;
  int acc = 0;
  if (npairs > 0 && c < candidate_limit(pp, npairs)) {
    double u1, u2, w;
    acc = candidate(pp.dc->x, c, &u1, &u2, &w) ? 1 : 0;
  }
  if (c < pp.ncand) pp.cand_flag[c] = acc;
  const int cnt = __popc(__ballot_sync(0xffffffffu, acc));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int q = 0; q < D_BS / 32; q++) s += sh[q];
    pp.cand_bsum[blockIdx.x] = s;
  }
}

// Accepted candidate number g (in stream order) becomes pair g.  The
// blocks' counts are summed here: only the blocks below the candidate limit
// have any (a handful), and each of those adds the counts before it; block 0
// also checks that the candidates cover the pairs needed -- never silently
// wrong: the step stops with an error status.
__global__ void __launch_bounds__(D_BS) k_rng_scatter(KP k, PP pp, int nb)
{
  fb_grid_dependency();
  __shared__ int wc[D_BS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int npairs = pp.dc->npairs;
  // sum of the counts of blocks [0, upto): every thread gets it
  auto block_count = [&](int upto) -> int {
    int v = 0;
    for (int q = threadIdx.x; q < upto; q += D_BS) v += pp.cand_bsum[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) wc[w] = v;
    __syncthreads();
    int t = 0;
    for (int q = 0; q < D_BS / 32; q++) t += wc[q];
    __syncthreads();
    return t;
  };
  if (blockIdx.x == 0) {
    const int total = block_count(nb);
    if (threadIdx.x == 0 && npairs > total) {
      pp.dc->err = 1;
      k.ctl->status = FB_ERR_INVALID;
    }
  }
  const long long c0 = (long long)blockIdx.x * D_BS;
  if (npairs <= 0 || c0 >= candidate_limit(pp, npairs)) return;  // no accepted candidate here
  const int prefix = block_count(blockIdx.x);
  const long long c = c0 + threadIdx.x;
  const int acc = (c < pp.ncand) ? pp.cand_flag[c] : 0;
  const unsigned b = __ballot_sync(0xffffffffu, acc);
  if (lane == 0) wc[w] = __popc(b);
  __syncthreads();
  int off = 0;
  for (int q = 0; q < w; q++) off += wc[q];
  const int g = prefix + off + __popc(b & ((1u << lane) - 1u));
  if (acc && g < npairs) {
    double u1, u2, ww;
    candidate(pp.dc->x, c, &u1, &u2, &ww);
    const double mult = sqrt((-2.0 * log(ww)) / ww);
    pp.pairs[g] = make_double2(u1 * mult, u2 * mult);
    if (g == npairs - 1) pp.dc->c_last = c;
  }
}

// Minimum_Stopping_Time (Dsys.c:757-759), the smallest stopping time of the
// substep (the dust time-step bound).  Non-negative doubles order like their
// bit patterns, so an integer minimum on the bits is a minimum on the
// values, exact in any order: the lanes that get here together first take their
// minimum (high words, then low words among the lanes with the smallest
// high word), and one of them updates the global value -- one atomic per
// warp instead of one per particle, all on the same address.
static __device__ __forceinline__ void record_stopping_time(const PP &pp, double Ts)
{
  const unsigned m = __activemask();
  const unsigned long long v = (Ts >= 0.0) ? (unsigned long long)__double_as_longlong(Ts) : ~0ull;
  const unsigned hi = (unsigned)(v >> 32), lo = (unsigned)v;
  const unsigned mh = __reduce_min_sync(m, hi);
  const unsigned ml = __reduce_min_sync(m, (hi == mh) ? lo : 0xffffffffu);
  const unsigned long long w = ((unsigned long long)mh << 32) | ml;
  if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && w != ~0ull) atomicMin((long long *)&pp.dc->min_ts, (long long)w);
}

// ----------------------------------- 4. kicks, interpolation, velocities
// mode 0: one substep (kick, interpolation, UpdateDustVelocities, and the
// second interpolation of SourceEuler.c:529-530 when WRITEDUSTDENSITY);
// mode 1: the interpolation call of main.c:287 (Stokes numbers only).
__global__ void __launch_bounds__(D_BS, 3) k_dust_update(KP k, PP pp, int mode)
{
  fb_grid_dependency();
  const int q = blockIdx.x * D_BS + threadIdx.x;  // storage slot
  if (q >= pp.n) return;
  // a candidate shortfall (k_rng_scatter) leaves pairs unset: the substep's
  // particles are not advanced, the step stops with an error status and
  // fb_dust_download refuses the state from then on
  if (mode == 0 && pp.dc->err) return;
  const int qr = (mode == 0) ? pp.orig[q] : 0;  // the reference's index: kick flag and rank
  const int ns = k.ns, nr = k.nr;
  const double rinf0 = k.rinf[0], rsupl = k.rsup[nr - 1];
  double r = pp.r[q], th = pp.th[q];
  // ---- turbulent kick (DustUpdate.c:56-105, Charnoz et al. 2011 eq. 21)
  if (mode == 0 && pp.flag[qr]) {
    const double timestep = 2.0 * k.ctl->dt;
    const double St = pp.st[q];
    const double visc = viscosity_at(k, pp, r);
    const double D_dust = visc * (1.0 + 4.0 * (St * St)) * powm2(1. + St * St);
    // `while (r >= Rinf[ip] && ip <= nr-1) ip++; ip--` (r >= Rinf[0] here)
    const int ip = last_not_above(pp, k.rinf, nr, r);
    int jp = (int)floor(ns * (th - pp.aziinf0) / (pp.azisupl - pp.aziinf0));
    if (jp == ns) jp = 0;
    jp = min(max(jp, 0), ns - 1);
    const size_t lp = (size_t)ip * ns + jp;
    const size_t lpm1 = (ip != 0) ? lp - ns : lp;
    const size_t lpjm = (jp == 0) ? (size_t)ip * ns + ns - 1 : lp - 1;
    // this particle's deviates (see the head of the file)
    const fb_dust_ctl *d = pp.dc;
    const long long M = d->kicks + pp.kidx[qr] + pp.kick_bsum[qr / SCAN_BS];
    const long long t = M / 2;
    const int odd = (int)(M & 1ll);
    double xr, xp;
    if (t < d->t_start) {
      xr = d->carry_rad;
      xp = d->carry_phi;
    } else {
      const long long e = t - d->t_start;
      const double2 pr = pp.pairs[2 * e], pf = pp.pairs[2 * e + 1];
      xr = odd ? pr.y : pr.x;
      xp = odd ? pf.y : pf.x;
    }
    const double dens_lp = k.rho[lp];
    const double dr_mean = D_dust / dens_lp * (dens_lp - k.rho[lpm1]) * k.invdiffrmed[ip] * timestep;
    const double sigma_r_squared = 2.0 * D_dust * timestep;
    r = r + (dr_mean + sqrt(sigma_r_squared) * xr);
    const double dxtheta = (k.pmax - k.pmin) / (double)ns * k.rmed[ip];
    const double invdxtheta = 1.0 / dxtheta;
    const double dphi_mean = D_dust / dens_lp * (dens_lp - k.rho[lpjm]) * invdxtheta * timestep / r;
    th = th + (dphi_mean + sqrt(sigma_r_squared) / r * xp);
    th = wrap_azimuth(pp, th);
    pp.r[q] = r;
    pp.th[q] = th;
  }
  if (!((r >= rinf0) && (r < rsupl))) return;
  // ---- 1) cell of the particle (Dsys.c:363-372)
  const double rp = r, tp = th;
  // `while (rp >= Rinf[ip]) ip++; ip--` with Rinf[0] <= rp < Rinf[nr]
  const int ip = last_not_above(pp, k.rinf, nr + 1, rp);
  int jp = (int)floor(ns * (tp - pp.aziinf0) / (pp.azisupl - pp.aziinf0));
  if (jp == ns) jp = 0;
  jp = min(max(jp, 0), ns - 1);
  const double delta_phi = pp.delta_phi, delta_r = pp.delta_r;
  const double rdelta_phi = 1.0 / delta_phi, rdelta_r = 1.0 / delta_r;
  const int want_sg = k.self_gravity && pp.feel_sg;
  double vrg = 0.0, rgp = 0.0, rind = 0.0, rsg = 0.0;
  double vtg = 0.0, agp = 0.0, aind = 0.0, asg = 0.0;
  double densg = 0.0, csg = 0.0;
  // The stencils' weights: radial ones at Rinf (2a) and Rmed (2b, 2c),
  // azimuthal ones at the cell centres (2a, 2c) and interfaces (2b); each
  // is computed once and reused, as the same values enter the sums.
  double wr_inf[3], wr_med[3], wt_c[3], wt_i[3];
  int jc[3], ji[3];
#if FB_FAST
  // one logarithm per particle: |log(rp / R)| as |log rp - log R|
  const double lrp = pp.log_grid ? log(rp) : 0.0;
#endif
#pragma unroll
  for (int t = 0; t < 3; t++) {
    const int i = ip - 1 + t;
    if (i >= 0 && i <= nr - 1) {
#if FB_FAST
      wr_inf[t] = tsc_weight(pp.log_grid ? fabs(lrp - pp.log_rinf[i]) : fabs(rp - k.rinf[i]), delta_r, rdelta_r);
      wr_med[t] = tsc_weight(pp.log_grid ? fabs(lrp - pp.log_rmed[i]) : fabs(rp - k.rmed[i]), delta_r, rdelta_r);
#else
      wr_inf[t] = tsc_weight(pp.log_grid ? fabs(log(fb_quot(rp, k.rinf[i], k.invrinf[i]))) : fabs(rp - k.rinf[i]),
                             delta_r, rdelta_r);
      wr_med[t] = tsc_weight(pp.log_grid ? fabs(log(fb_quot(rp, k.rmed[i], k.invrmed[i]))) : fabs(rp - k.rmed[i]),
                             delta_r, rdelta_r);
#endif
    } else {
      wr_inf[t] = wr_med[t] = 0.0;
    }
    const int j = jp - 1 + t;
    double az;
    if (j >= 0 && j < ns) { jc[t] = j; az = pp.azimuth[j]; }
    else if (j < 0) { jc[t] = j + ns; az = pp.azimuth[0] + j * delta_phi; }
    else { jc[t] = j - ns; az = pp.azimuth[ns - 1] + (j + 1 - ns) * delta_phi; }
    wt_c[t] = tsc_weight(fabs(tp - az), delta_phi, rdelta_phi);
  }
  {
    const int myjp = (tp > pp.azimuth[jp]) ? jp + 1 : jp;
#pragma unroll
    for (int t = 0; t < 3; t++) {
      const int j = myjp - 1 + t;
      double az;
      if (j >= 0 && j < ns) { ji[t] = j; az = pp.aziinf[j]; }
      else if (j < 0) { ji[t] = j + ns; az = pp.aziinf[0] + j * delta_phi; }
      else { ji[t] = j - ns; az = pp.aziinf[ns - 1] + (j + 1 - ns) * delta_phi; }
      wt_i[t] = tsc_weight(fabs(tp - az), delta_phi, rdelta_phi);
    }
  }
  // ---- 2a) vrad-staggered values: (Rinf[i], Azimuth[j]) (Dsys.c:397-487)
#pragma unroll
  for (int tj = 0; tj < 3; tj++) {
    const double wt = wt_c[tj];
#pragma unroll
    for (int ti = 0; ti < 3; ti++) {
      const int i = ip - 1 + ti;
      if (i < 0 || i > nr - 1) continue;
      const double wr = wr_inf[ti];
      const size_t l = (size_t)i * ns + jc[tj];
      vrg += (wr * wt * k.vr[l]);
      rgp += (wr * wt * k.rgp[l]);
      if (k.indirect_term) rind += (wr * wt * k.rind[l]);
      if (want_sg) rsg += (wr * wt * k.rsga[l]);
    }
  }
  // ---- 2b) vtheta-staggered values: (Rmed[i], AziInf[j]) (Dsys.c:510-588);
  // the reference adds Rmed*OmegaFrame to vtheta around the call, and the
  // supported frame is non-rotating (OmegaFrame = 0)
#pragma unroll
  for (int tj = 0; tj < 3; tj++) {
    const double wt = wt_i[tj];
#pragma unroll
    for (int ti = 0; ti < 3; ti++) {
      const int i = ip - 1 + ti;
      if (i < 0 || i > nr - 1) continue;
      const double wr = wr_med[ti];
      const size_t l = (size_t)i * ns + ji[tj];
      vtg += (wr * wt * k.vt[l]);
      agp += (wr * wt * k.agp[l]);
      if (k.indirect_term) aind += (wr * wt * k.aind[l]);
      if (want_sg) asg += (wr * wt * k.asga[l]);
    }
  }
  // ---- 2c) cell-centred values: (Rmed[i], Azimuth[j]) (Dsys.c:617-711).
  // The dust deposit of this loop is Particles_Mass times the weights; the
  // particle mass is zero without a dust fluid (main.c:187-200), so there
  // is nothing to deposit.
#pragma unroll
  for (int tj = 0; tj < 3; tj++) {
    const double wt = wt_c[tj];
#pragma unroll
    for (int ti = 0; ti < 3; ti++) {
      const int i = ip - 1 + ti;
      if (i < 0 || i > nr - 1) continue;
      const double wr = wr_med[ti];
      const size_t l = (size_t)i * ns + jc[tj];
      densg += (wr * wt * k.rho[l]);
      csg += (wr * wt * k.cs[l]);
    }
  }
  const double size = pp.size[q];
  const double vrd = pp.vr[q], vtd = pp.vth[q];
  const double St = stokes_number(pp, size, rp, vrd, vtd, vrg, vtg, csg, densg);
  if (mode == 1) {
    pp.st[q] = St;
    record_stopping_time(pp, St * pow15(rp));
    return;
  }
  // ---- UpdateDustVelocities (DustUpdate.c:301-428), first-order integrator
  const double dt = k.ctl->dt;
  const double rd = rp, td = tp;
  int LocalDustFeelDisk = pp.feel_disk;
  if ((rd < pp.rmin) || (rd > pp.rmax)) LocalDustFeelDisk = 0;
  const double rp15 = pow15(rd);
  const double stoptime = St * rp15;
  double vr_new, vth_new;
  if ((stoptime < dt) && pp.sfta) {
    // short-friction-time approximation
    vr_new = vrg + stoptime * rgp / densg;
    vth_new = vtg + stoptime * agp / densg;
    pp.l[q] = rd * vth_new;
  } else {
    // semi-implicit integrator
    double FgravR = -powm2(rd);
    double FgravTh = 0.;
    if ((fabs(FgravR + vtd * vtd / rd) < 1e-15) && (!pp.feel_planets) && (!pp.feel_disk) && (!pp.feel_sg))
      FgravR = -vtd * vtd / rd;
    if (pp.feel_planets) {
      const fb_ctl *c = k.ctl;
      const fb_dust_ctl *dc = pp.dc;  // radius, azimuth, smoothing from k_planets
      for (int p = 0; p < c->np; p++) {
        const double rpl = dc->pl_r[p], tpl = dc->pl_t[p], eps = dc->pl_eps[p];
        const double mp = c->pm[p];
        const double cdt = cos(td - tpl), d = sqrt(rd * rd + rpl * rpl - 2.0 * rd * rpl * cdt + eps * eps);
        const double d3 = powm3(d);
        FgravR += mp * (rpl * cdt - rd) * d3;
        FgravTh += -mp * rpl * sin(td - tpl) * d3;
      }
    }
    if (k.indirect_term) {
      FgravR += rind;
      FgravTh += aind;
    }
    if (k.self_gravity && pp.feel_sg) {
      FgravR += rsg;
      FgravTh += asg;
    }
    const double den = 1.0 + LocalDustFeelDisk * dt / stoptime;
    const double numTh = (vtd - vtg) + dt * (FgravTh - vrd * vtd / rd);
    vth_new = vtg + numTh / den;
    const double numR = (vrd - vrg) + dt * (FgravR + (vth_new * vth_new) / rd);
    vr_new = vrg + numR / den;
  }
  pp.vr[q] = vr_new;
  pp.vth[q] = vth_new;
  // the interpolation after RotateDsys recomputes the Stokes number with the
  // updated velocities; the next substep's kick uses that one
  const double St_out = pp.restokes ? stokes_number(pp, size, rp, vr_new, vth_new, vrg, vtg, csg, densg) : St;
  pp.st[q] = St_out;
  record_stopping_time(pp, pp.restokes ? St_out * rp15 : stoptime);
}

// ----------------------------------------------------- 5. bookkeeping
__global__ void k_dust_finish(PP pp)
{
  fb_grid_dependency();
  fb_dust_ctl *d = pp.dc;
  const long long G = d->kicks, K = d->K;
  if (d->err) {  // the stream position is unknown after a shortfall: leave it
    d->K = 0;
    d->npairs = 0;
    return;
  }
  if (d->npairs > 0) d->x = lcg_skip(d->x, (unsigned long long)(2 * (d->c_last + 1)));
  if (K > 0 && ((G + K) & 1ll)) {
    // an odd number of calls in total: each generator keeps the second
    // deviate of its last pair for its next call
    const long long e = (G + K - 1) / 2 - d->t_start;
    if (e >= 0) {
      d->carry_rad = pp.pairs[2 * e].y;
      d->carry_phi = pp.pairs[2 * e + 1].y;
    }
  }
  d->kicks = G + K;
  d->K = 0;
  d->npairs = 0;
}

// ------------------------------------------------------ 6. cell sort
// Counting sort of the particles by cell (once per DT): key = ip*ns + jp of
// the particles on the grid, nr*ns for the others.
__global__ void __launch_bounds__(D_BS) k_cell_key(KP k, PP pp)
{
  fb_grid_dependency();
  const int q = blockIdx.x * D_BS + threadIdx.x;
  if (q >= pp.n) return;
  const double r = pp.r[q], th = pp.th[q];
  const int nr = k.nr, ns = k.ns;
  int key = nr * ns;
  if (r >= k.rinf[0] && r < k.rsup[nr - 1]) {
    const int ip = last_not_above(pp, k.rinf, nr + 1, r);
    int jp = (int)floor(ns * (th - pp.aziinf0) / (pp.azisupl - pp.aziinf0));
    jp = min(max(jp, 0), ns - 1);
    key = ip * ns + jp;
  }
  pp.key[q] = key;
  atomicAdd(pp.cell_count + key, 1);
}

// exclusive block offsets -> global offsets
__global__ void __launch_bounds__(SCAN_BS) k_scan_add(int *v, const int *bsum, int n)
{
  fb_grid_dependency();
  const int g = blockIdx.x * SCAN_BS + threadIdx.x;
  if (g < n) v[g] += bsum[blockIdx.x];
}

__global__ void __launch_bounds__(SCAN_BS) k_scan_top_only(int *blocksum, int nb) {
  fb_grid_dependency(); scan_top(blocksum, nb); }

__global__ void __launch_bounds__(D_BS) k_cell_scatter(PP pp)
{
  fb_grid_dependency();
  const int q = blockIdx.x * D_BS + threadIdx.x;
  if (q >= pp.n) return;
  const int pos = atomicAdd(pp.cell_count + pp.key[q], 1);  // the offsets, consumed as cursors
  pp.perm[pos] = q;
}

// Moves the particles into the sorted order: slot t takes old slot perm[t].
__global__ void __launch_bounds__(D_BS) k_cell_gather(PP pp)
{
  fb_grid_dependency();
  const int t = blockIdx.x * D_BS + threadIdx.x;
  if (t >= pp.n) return;
  const int s = pp.perm[t];
  const size_t n = pp.n;
  double *x = pp.pscratch;
  x[t] = pp.r[s];
  x[n + t] = pp.th[s];
  x[2 * n + t] = pp.vr[s];
  x[3 * n + t] = pp.vth[s];
  x[4 * n + t] = pp.l[s];
  x[5 * n + t] = pp.size[s];
  x[6 * n + t] = pp.st[s];
  pp.oscratch[t] = pp.orig[s];
}

__global__ void __launch_bounds__(D_BS) k_cell_copy(PP pp)
{
  fb_grid_dependency();
  const int t = blockIdx.x * D_BS + threadIdx.x;
  if (t >= pp.n) return;
  const size_t n = pp.n;
  const double *x = pp.pscratch;
  pp.r[t] = x[t];
  pp.th[t] = x[n + t];
  pp.vr[t] = x[2 * n + t];
  pp.vth[t] = x[3 * n + t];
  pp.l[t] = x[4 * n + t];
  pp.size[t] = x[5 * n + t];
  pp.st[t] = x[6 * n + t];
  pp.orig[t] = pp.oscratch[t];
}

int fb_launch_dust_sort(const KP &k, const PP &pp, cudaStream_t s)
{
  const int nb = (pp.n + D_BS - 1) / D_BS, nc = pp.ncells, ncb = (nc + SCAN_BS - 1) / SCAN_BS;
  cudaMemsetAsync(pp.cell_count, 0, (size_t)nc * sizeof(int), s);
  fb_launch(k_cell_key, nb, D_BS, 0, s, k, pp);
  fb_launch(k_scan_block, ncb, SCAN_BS, 0, s, pp.cell_count, pp.cell_count, pp.cell_bsum, nc);
  fb_launch(k_scan_top_only, 1, SCAN_BS, 0, s, pp.cell_bsum, ncb);
  fb_launch(k_scan_add, ncb, SCAN_BS, 0, s, pp.cell_count, pp.cell_bsum, nc);
  fb_launch(k_cell_scatter, nb, D_BS, 0, s, pp);
  fb_launch(k_cell_gather, nb, D_BS, 0, s, pp);
  fb_launch(k_cell_copy, nb, D_BS, 0, s, pp);
  return 7;
}

// storage slots in the reference's order (after an upload)
__global__ void __launch_bounds__(D_BS) k_iota(int *v, int n)
{
  fb_grid_dependency();
  const int t = blockIdx.x * D_BS + threadIdx.x;
  if (t < n) v[t] = t;
}
void fb_launch_dust_iota(const PP &pp, cudaStream_t s)
{
  fb_launch(k_iota, (pp.n + D_BS - 1) / D_BS, D_BS, 0, s, pp.orig, pp.n);
}

// dst[orig[t]] = src[t]: one particle array back in the reference's order
__global__ void __launch_bounds__(D_BS) k_to_reference_order(const int *orig, const double *src, double *dst, int n)
{
  fb_grid_dependency();
  const int t = blockIdx.x * D_BS + threadIdx.x;
  if (t < n) dst[orig[t]] = src[t];
}
void fb_launch_dust_to_reference_order(const PP &pp, const double *src, double *dst, cudaStream_t s)
{
  fb_launch(k_to_reference_order, (pp.n + D_BS - 1) / D_BS, D_BS, 0, s, pp.orig, src, dst, pp.n);
}

// ---------------------------------------------------------- launchers
int fb_dust_launches(const PP &pp) { return pp.feel_turb ? 7 : 2; }

void fb_launch_dust_substep(const KP &k, const PP &pp, cudaStream_t s, cudaEvent_t planets_done)
{
  const int nb = (pp.n + D_BS - 1) / D_BS;
  fb_launch(k_dust_drift, nb, D_BS, 0, s, k, pp);
  if (pp.feel_turb) {
    const int nsb = (pp.n + SCAN_BS - 1) / SCAN_BS;
    fb_launch(k_scan_block, nsb, SCAN_BS, 0, s, pp.flag, pp.kidx, pp.kick_bsum, pp.n);
    fb_launch(k_kick_top, 1, SCAN_BS, 0, s, pp, nsb);
    const int ncb = (pp.ncand + D_BS - 1) / D_BS;
    fb_launch(k_rng_count, ncb, D_BS, 0, s, pp);
    fb_launch(k_rng_scatter, ncb, D_BS, 0, s, k, pp, ncb);
  }
  if (planets_done) cudaStreamWaitEvent(s, planets_done, 0);  // positions after the planets' step
  fb_launch(k_dust_update, nb, D_BS, 0, s, k, pp, 0);
  if (pp.feel_turb) fb_launch(k_dust_finish, 1, 1, 0, s, pp);
}

void fb_launch_dust_interpolation_only(const KP &k, const PP &pp, cudaStream_t s)
{
  const int nb = (pp.n + D_BS - 1) / D_BS;
  fb_launch(k_dust_update, nb, D_BS, 0, s, k, pp, 1);
}
