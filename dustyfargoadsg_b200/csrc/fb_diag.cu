// fb_diag.cu -- disc diagnostics with no counterpart in the reference (it has
// no vortensity routine): vortensity on the staggered grid and azimuthal
// means, used to compare coarse runs with fine ones.
//
// Vortensity at the cell corner (R_inf[i], phi_inf[j]), i = 1 .. nr-1, where
// vtheta (at R_med, phi_inf) and vrad (at R_inf, phi_med) are both one
// half-cell away:
//   omega_z = [ (R_med[i] vt[i,j] - R_med[i-1] vt[i-1,j]) / (R_med[i] - R_med[i-1])
//             - (vr[i,j] - vr[i,j-1]) / dphi ] / R_inf[i]  +  2 OmegaFrame
//   Sigma_c = (Sigma[i,j] + Sigma[i-1,j] + Sigma[i,j-1] + Sigma[i-1,j-1]) / 4
//   xi      = omega_z / Sigma_c
// Ring 0 and ring nr are zero.  Azimuthal means use one CTA per ring and a
// fixed reduction order, so they are bit-reproducible.
#include <cuda_runtime.h>
#include "fb_dev.cuh"

#define DG_BS 256

__global__ void __launch_bounds__(DG_BS) k_vortensity(KP k, double *xi)
{
  const int i = blockIdx.y, ns = k.ns;
  const int j = blockIdx.x * DG_BS + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j;
  if (i == 0) {
    xi[l] = 0.0;
    return;
  }
  const size_t lim = l - ns;
  const size_t ljm = (j == 0) ? (size_t)i * ns + ns - 1 : l - 1;
  const size_t limjm = ljm - ns;
  const double drvt = (k.rmed[i] * k.vt[l] - k.rmed[i - 1] * k.vt[lim]) / (k.rmed[i] - k.rmed[i - 1]);
  const double dvr = (k.vr[l] - k.vr[ljm]) * k.invdphi;
  const double omega = (drvt - dvr) / k.rinf[i] + 2.0 * omf(k);
  const double sig = 0.25 * (k.rho[l] + k.rho[lim] + k.rho[ljm] + k.rho[limjm]);
  xi[l] = omega / sig;
}

// mean over the ns entries of each ring of f (one CTA per ring)
__global__ void __launch_bounds__(DG_BS) k_ring_mean(const double *f, int ns, double *out)
{
  __shared__ double sh[DG_BS];
  const int i = blockIdx.x;
  double s = 0.0;
  for (int j = threadIdx.x; j < ns; j += DG_BS) s += f[(size_t)i * ns + j];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = DG_BS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[i] = sh[0] / (double)ns;
}

void fb_launch_vortensity(const KP &k, double *xi, cudaStream_t s)
{
  dim3 g((k.ns + DG_BS - 1) / DG_BS, k.nr);
  k_vortensity<<<g, DG_BS, 0, s>>>(k, xi);
}

void fb_launch_ring_mean(const double *f, int nr, int ns, double *out, cudaStream_t s)
{
  k_ring_mean<<<nr, DG_BS, 0, s>>>(f, ns, out);
}

// ComputeForce (Force.c:77-253) of the disc on a body at (x, y), for the
// planet logs of the reference's loop (UpdateLog, Force.c:266-328): one CTA
// per ring sums G m_cell d / (d^2 + eps^2)^(3/2) over the ring's cells, without
// (k = 0) and with (k = 1) the Hill cut at `cutoff` (EXCLUDEHILLFACTOR times
// the Hill radius, dimfxy = 2), each term in the reference's expression order;
// part[4 i ..] = fx(k=0), fx(k=1), fy(k=0), fy(k=1) of ring i.  The host adds
// the rings in order into the inner and outer sums.
__global__ void __launch_bounds__(DG_BS) k_body_force(KP k, double x, double y, double rsmoothing,
                                                      double cutoff, double *part)
{
  __shared__ double sh[4][DG_BS];
  const int i = blockIdx.x, ns = k.ns;
  const double rmi = k.rmed[i], surf = k.surf[i];
  double f[4] = {0.0, 0.0, 0.0, 0.0};
  for (int j = threadIdx.x; j < ns; j += DG_BS) {
    const size_t l = (size_t)i * ns + j;
    const double xc = rmi * k.cosaz[j], yc = rmi * k.sinaz[j];
    const double cellmass = surf * k.rho[l];
    const double dx = xc - x, dy = yc - y;
    const double d2 = dx * dx + dy * dy;
    const double planet_distance = sqrt(d2);
    const double dist2 = d2 + rsmoothing * rsmoothing;
    const double distance = sqrt(dist2);
    const double InvDist3 = 1.0 / dist2 / distance;
    double hill_cut;
    if (planet_distance / cutoff < 0.5) {
      hill_cut = 0.0;
    } else if (planet_distance > cutoff) {
      hill_cut = 1.0;
    } else {
      const double s = sin((planet_distance / cutoff - .5) * M_PI);
      hill_cut = s * s;  // pow(., 2.)
    }
    f[0] += FB_G * cellmass * dx * InvDist3 * 1.0;
    f[1] += FB_G * cellmass * dx * InvDist3 * hill_cut;
    f[2] += FB_G * cellmass * dy * InvDist3 * 1.0;
    f[3] += FB_G * cellmass * dy * InvDist3 * hill_cut;
  }
#pragma unroll
  for (int q = 0; q < 4; q++) sh[q][threadIdx.x] = f[q];
  __syncthreads();
  for (int w = DG_BS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int q = 0; q < 4; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) part[(size_t)i * 4 + threadIdx.x] = sh[threadIdx.x][0];
}

void fb_launch_body_force(const KP &k, double x, double y, double rsmoothing, double cutoff, double *part,
                          cudaStream_t s)
{
  k_body_force<<<k.nr, DG_BS, 0, s>>>(k, x, y, rsmoothing, cutoff, part);
}
