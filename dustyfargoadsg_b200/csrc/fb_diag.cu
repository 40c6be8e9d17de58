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
  const double omega = (drvt - dvr) / k.rinf[i] + 2.0 * k.omega_frame;
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
