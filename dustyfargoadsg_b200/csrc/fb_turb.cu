// fb_turb.cu -- the stochastic turbulent potential of Laughlin, Steinacker &
// Adams (2004) as modified by Baruteau & Lin (2010): ApplyLSAOnPotential
// (src/turb.c:13-135), called by FillForcesArrays at every substep
// (src/Pframeforce.c:125-128) when MHD is L.
//
// Per substep, at the substep's starting time t (PhysicalTime before the
// substep's dt is added):
//  1. k_lsa_modes, one CTA: thread 0 redraws, in mode order, every mode whose
//     lifetime has ended (t >= tf) from the drand48 stream, exactly as the
//     reference's first loop does (turb.c:30-72: m from m^2 uniform in
//     [4, (nsec/2)^2], rc uniform in [TURBRMIN, TURBRMAX], phic uniform in
//     [0, PMAX-PMIN), xi by Marsaglia's polar method); then one thread per
//     mode sets the redrawn modes' omegac, sigma, deltat, t0, tf (turb.c:
//     85-93) and every mode's time factor sin(pi ttilde / deltat) and phase
//     P = phic + (omegac - OmegaFrame) ttilde.  The draws are integer-exact
//     and their arithmetic is written without contraction, so the GPU
//     consumes the reference's stream and draws the same integers m.
//  2. k_lsa_tables, one CTA per redrawn mode: its azimuthal factors
//     cos(m Azimuth[j]) and sin(m Azimuth[j]) and its radial envelope
//     mygamma(r)/r xi exp(-(r-rc)^2/sigma^2) per ring (turb.c:118-126).
//  3. k_lsa_add, after k_potential: Pot[l] += ampl cos(m Azimuth[j] - P) for
//     the active modes in mode order (turb.c:127-131), evaluated as
//     A cos(m Azimuth) + B sin(m Azimuth) with A = ampl cos P, B = ampl sin P.
//     Each CTA holds A and B of its rings in shared memory and each thread a
//     column of R rings in registers, so a cell costs two multiply-adds per
//     mode.  The reference evaluates cos of the whole argument (up to ~1e4
//     radians, rounded to ~1e-12 absolute before the cosine); the two forms
//     differ by that rounding times the amplitude (~1e-5 of the potential),
//     far below the parity bar.
#include <math.h>
#include "fb_dev.cuh"

static __device__ __forceinline__ double lsa_u48(unsigned long long &x)
{
  x = (0x5DEECE66Dull * x + 0xBull) & 0xFFFFFFFFFFFFull;
  return (double)x * 0x1p-48;  // drand48: the 48 bits as a fraction, exact
}

#define LSA_MAX_TRIES 100000  // Marsaglia candidates per deviate (acceptance pi/4)

__global__ void __launch_bounds__(256) k_lsa_modes(KP k)
{
  fb_grid_dependency();
  fb_lsa *L = k.lsa_st;
  const double t = k.ctl->t_sub;
  const int nm = k.lsa_nm;
  if (threadIdx.x == 0) {
    unsigned long long x = L->x;
    const double m_min = 2.0, m_max = (double)k.ns / 2.0;
    const double m2span = __dsub_rn(__dmul_rn(m_max, m_max), __dmul_rn(m_min, m_min));
    for (int q = 0; q < nm; q++) {
      const int rd = (t >= L->tf[q]) ? 1 : 0;
      L->redraw[q] = rd;
      if (!rd) continue;
      // m^2 uniform between m_min^2 and m_max^2 (turb.c:52-55)
      L->m[q] = (int)(long)sqrt(__dadd_rn(__dmul_rn(m_min, m_min), __dmul_rn(m2span, lsa_u48(x))));
      L->rc[q] = __dadd_rn(k.lsa_rmin, __dmul_rn(__dsub_rn(k.lsa_rmax, k.lsa_rmin), lsa_u48(x)));
      L->phic[q] = __dmul_rn(k.pmax - k.pmin, lsa_u48(x));
      double x1 = 0.0, w = 1.0;
      int tries = 0;
      do {
        x1 = __dsub_rn(__dmul_rn(2.0, lsa_u48(x)), 1.0);
        const double x2 = __dsub_rn(__dmul_rn(2.0, lsa_u48(x)), 1.0);
        w = __dadd_rn(__dmul_rn(x1, x1), __dmul_rn(x2, x2));
      } while (w >= 1.0 && ++tries < LSA_MAX_TRIES);
      if (w >= 1.0) {  // cannot happen with this generator; never loop forever
        L->status = FB_ERR_INVALID;
        k.ctl->status = FB_ERR_INVALID;
        w = 0.5;
      }
      w = sqrt((-2.0 * log(w)) / w);
      L->xi[q] = x1 * w;
    }
    L->x = x;
    // the modes that add to the potential (turb.c:116)
    int na = 0;
    for (int q = 0; q < nm; q++)
      if (L->m[q] <= 6 || !k.lsa_highm) L->act[na++] = q;
    L->nact = na;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nm; q += blockDim.x) {
    if (L->redraw[q]) {  // turb.c:85-93
      const double rc = L->rc[q], m = (double)L->m[q];
      L->omegac[q] = pow(rc, -1.5);
      L->sigma[q] = M_PI * rc / 4.0 / m;
      L->deltat[q] = k.lsa_speedup * 2.0 * M_PI * rc / m / sqrt(m) / k.aspectratio / pow(rc, -0.5 + k.flaringindex);
      L->t0[q] = t;
      L->tf[q] = t + L->deltat[q];
    }
    const double ttilde = t - L->t0[q];
    L->s[q] = sin(M_PI * ttilde / L->deltat[q]);
    const double P = L->phic[q] + (L->omegac[q] - omf(k)) * ttilde;
    double sp, cp;
    sincos(P, &sp, &cp);
    L->cp[q] = cp;
    L->sp[q] = sp;
  }
}

// blockIdx.x = mode; only redrawn modes recompute their tables
__global__ void __launch_bounds__(256) k_lsa_tables(KP k)
{
  fb_grid_dependency();
  const fb_lsa *L = k.lsa_st;
  const int q = blockIdx.x, ns = k.ns, nr = k.nr;
  if (!L->redraw[q]) return;
  const double m = (double)L->m[q];
  double *cs = k.lsa_cs + (size_t)q * ns, *sn = k.lsa_cs + ((size_t)k.lsa_nm + q) * ns;
  for (int j = threadIdx.x; j < ns; j += blockDim.x) {
    const double angle = k.pmin + (k.pmax - k.pmin) * (double)j / (double)ns;  // Azimuth[j], SourceEuler.c:163
    double s, c;
    sincos(m * angle, &s, &c);
    cs[j] = c;
    sn[j] = s;
  }
  // radial envelope (turb.c:118-126) without the time factor; the cavity
  // profile of the amplitude with its defaults (rmin < 0 < r, ratio 1) is
  // mygamma = gamma everywhere
  const double rc = L->rc[q], sigma = L->sigma[q], xi = L->xi[q];
  for (int i = threadIdx.x; i < nr; i += blockDim.x) {
    const double r = k.rmed[i];
    double mygamma = k.lsa_gamma;
    if (r < k.cav_rmin) mygamma = k.lsa_gamma * k.cav_ratio;
    if ((r >= k.cav_rmin) && (r <= k.cav_rmax))
      mygamma = k.lsa_gamma * exp((k.cav_rmax - r) / (k.cav_rmax - k.cav_rmin) * log(k.cav_ratio));
    if (r > k.cav_rmax) mygamma = k.lsa_gamma;
    k.lsa_g[(size_t)q * nr + i] = mygamma / r * xi * exp(-(r - rc) * (r - rc) / sigma / sigma);
  }
}

#define LSA_R 8     // rings per thread
#define LSA_T 128   // columns per CTA

__global__ void __launch_bounds__(LSA_T) k_lsa_add(KP k)
{
  fb_grid_dependency();
  __shared__ double2 ab[LSA_R][FB_LSA_MAX_MODES];  // (A, B) of each ring and active mode
  const fb_lsa *L = k.lsa_st;
  const int ns = k.ns, nr = k.nr, nact = L->nact;
  const int i0 = blockIdx.y * LSA_R, nrow = min(LSA_R, nr - i0);
  for (int idx = threadIdx.x; idx < nrow * nact; idx += blockDim.x) {
    const int r = idx / nact, a = idx - r * nact, q = L->act[a];
    const double ampl = k.lsa_g[(size_t)q * nr + i0 + r] * L->s[q];
    ab[r][a] = make_double2(ampl * L->cp[q], ampl * L->sp[q]);
  }
  __syncthreads();
  const int j = blockIdx.x * LSA_T + threadIdx.x;
  if (j >= ns) return;
  double acc[LSA_R];
#pragma unroll
  for (int r = 0; r < LSA_R; r++) acc[r] = (r < nrow) ? k.pot[(size_t)(i0 + r) * ns + j] : 0.0;
  const double *cs = k.lsa_cs, *sn = k.lsa_cs + (size_t)k.lsa_nm * ns;
  for (int a = 0; a < nact; a++) {
    const int q = L->act[a];
    const double c = cs[(size_t)q * ns + j], s = sn[(size_t)q * ns + j];
#pragma unroll
    for (int r = 0; r < LSA_R; r++) {
      const double2 v = ab[r][a];
      acc[r] += v.x * c + v.y * s;
    }
  }
#pragma unroll
  for (int r = 0; r < LSA_R; r++)
    if (r < nrow) k.pot[(size_t)(i0 + r) * ns + j] = acc[r];
}

void fb_launch_lsa_modes(const KP &k, cudaStream_t s)
{
  fb_launch(k_lsa_modes, 1, 256, 0, s, k);
  fb_launch(k_lsa_tables, k.lsa_nm, 256, 0, s, k);
}

void fb_launch_lsa_add(const KP &k, cudaStream_t s)
{
  fb_launch(k_lsa_add, dim3((k.ns + LSA_T - 1) / LSA_T, (k.nr + LSA_R - 1) / LSA_R), LSA_T, 0, s, k);
}
