// fb_closure.cu -- learned coarse-grid closure (no counterpart in the
// reference): a 4-layer periodic-in-azimuth CNN (3x3 convolutions, 32
// channels, GELU) that reads a coarse disc (Sigma, vrad, vtheta, potential)
// and predicts flux corrections for mass, angular momentum and radial
// momentum; the corrections are applied as flux differences, so the disc's
// mass and angular momentum change only by round-off.  Trained on the GPU by
// the kernels below against coarse-grained fine-grid runs.
//
// Precision: BF16 weights and activations, FP32 accumulation on the tensor
// cores (mma.m16n8k16, bf16 x bf16 -> f32), FP32 master weights and Adam,
// FP64 for the disc state and the corrections applied to it.
//
// Layout: activations NHWC, [sample][ring][azimuth][channel]; weights
// [out][tap][in] with tap = (dy+1)*3 + (dx+1).  Azimuth is periodic, the
// radial direction zero-padded.
//
// What the network corrects: the mass of every coarse cell, through two
// face fluxes per cell (Fr through its inner radial face, Ft through its
// lower azimuthal face), in units of scale * Sigma0(face) where Sigma0 is
// the disc's initial density profile (geometric mean of the two rings at a
// radial face):
//   dSigma(i,j) = [Fr(i,j) mr(i) - Fr(i+1,j) mr(i+1) + Ft(i,j) - Ft(i,j+1)] / Surf[i]
// with mr(i) = 1 on the interior radial faces 1..nr-1, so sum Surf dSigma = 0.
// The corrected mass carries its angular momentum: each vtheta face's
// control volume (half of the cells j-1 and j) exchanges, through its four
// boundaries, the mass fluxes of the cells averaged onto those boundaries
// times the upwind specific angular momentum R vtheta, so the staggered
// angular momentum J = (Sigma(i,j-1) + Sigma(i,j))/2 R vtheta(i,j) changes
// only by round-off and a uniform rotation is left unchanged.  vrad is not
// modified.  The training set stores the conservative quantities m, J, P of
// the targets; the loss uses m.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <vector>
#include "fb_dev.cuh"

#define CL_LAYERS 4
#define CL_C 32      // hidden channels
#define CL_CIN 16    // input feature channels (7 used)
#define CL_COUT 16   // output channels (2 used: the mass fluxes Fr, Ft)
#define CL_TILE 64   // pixels per CTA in the convolutions
#define CL_BS 128

typedef __nv_bfloat16 bf16;

static const int kLayerIn[CL_LAYERS] = {CL_CIN, CL_C, CL_C, CL_C};
static const int kLayerOut[CL_LAYERS] = {CL_C, CL_C, CL_C, CL_COUT};

// ------------------------------------------------------------ helpers
static __device__ __forceinline__ float gelu_f(float x)
{
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}
static __device__ __forceinline__ float gelu_grad_f(float x)
{
  // d/dx [x Phi(x)] = Phi(x) + x phi(x)
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

static __device__ __forceinline__ unsigned pack_bf16x2(float lo, float hi)
{
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned *>(&v);
}

static __device__ __forceinline__ void mma_bf16(float *d, const unsigned *a, const unsigned *b)
{
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ------------------------------------------------------------ convolution
// One CTA: CL_TILE consecutive azimuths of one ring of one sample, all COUT
// output channels.  4 warps x 16 pixels; per warp COUT/8 n-tiles.
// MODE 0: hidden layer forward: y = GELU(acc + b) -> bf16, pre-activation -> z (if z)
// MODE 1: last layer forward: acc + b -> f32
// MODE 2: backward data: acc * GELU'(zin) -> bf16 (weights transposed/flipped, no bias)
template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(CL_BS) k_conv(const bf16 *__restrict__ in, const bf16 *__restrict__ w,
                                                const float *__restrict__ bias, const float *__restrict__ zin,
                                                bf16 *__restrict__ outb, float *__restrict__ outf,
                                                float *__restrict__ zout, int nr, int ns)
{
  constexpr int HP = CIN + 8;             // padded pixel stride (elements)
  constexpr int KW = 9 * CIN + 8;         // padded weight row (elements)
  __shared__ __align__(16) bf16 halo[3][CL_TILE + 2][HP];
  __shared__ __align__(16) bf16 wsm[COUT][KW];
  const int j0 = blockIdx.x * CL_TILE, i = blockIdx.y, b = blockIdx.z;
  const int tid = threadIdx.x;
  // input halo: rings i-1..i+1, azimuths j0-1..j0+CL_TILE (periodic), 16-byte chunks
  constexpr int CH = CIN / 8;  // 16-byte chunks per pixel
  for (int t = tid; t < 3 * (CL_TILE + 2) * CH; t += CL_BS) {
    const int c = t % CH, px = (t / CH) % (CL_TILE + 2), r = t / (CH * (CL_TILE + 2));
    const int ii = i - 1 + r;
    int jj = j0 - 1 + px;
    jj = jj < 0 ? jj + ns : (jj >= ns ? jj - ns : jj);
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (ii >= 0 && ii < nr) v = *reinterpret_cast<const uint4 *>(in + (((size_t)b * nr + ii) * ns + jj) * CIN + c * 8);
    *reinterpret_cast<uint4 *>(&halo[r][px][c * 8]) = v;
  }
  constexpr int WCH = 9 * CIN / 8;
  for (int t = tid; t < COUT * WCH; t += CL_BS) {
    const int c = t % WCH, o = t / WCH;
    *reinterpret_cast<uint4 *>(&wsm[o][c * 8]) = *reinterpret_cast<const uint4 *>(w + (size_t)o * 9 * CIN + c * 8);
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, tg = lane & 3;
  const int m0 = warp * 16;
  constexpr int NT = COUT / 8;
  float acc[NT][4];
#pragma unroll
  for (int n = 0; n < NT; n++) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
  for (int tap = 0; tap < 9; tap++) {
    const int dy = tap / 3, dx = tap % 3;  // halo row and column offset (0..2)
#pragma unroll
    for (int c0 = 0; c0 < CIN; c0 += 16) {
      unsigned a[4];
      a[0] = *reinterpret_cast<const unsigned *>(&halo[dy][m0 + g + dx][c0 + tg * 2]);
      a[1] = *reinterpret_cast<const unsigned *>(&halo[dy][m0 + g + 8 + dx][c0 + tg * 2]);
      a[2] = *reinterpret_cast<const unsigned *>(&halo[dy][m0 + g + dx][c0 + 8 + tg * 2]);
      a[3] = *reinterpret_cast<const unsigned *>(&halo[dy][m0 + g + 8 + dx][c0 + 8 + tg * 2]);
      const int k0 = tap * CIN + c0;
#pragma unroll
      for (int n = 0; n < NT; n++) {
        unsigned bb[2];
        bb[0] = *reinterpret_cast<const unsigned *>(&wsm[n * 8 + g][k0 + tg * 2]);
        bb[1] = *reinterpret_cast<const unsigned *>(&wsm[n * 8 + g][k0 + 8 + tg * 2]);
        mma_bf16(acc[n], a, bb);
      }
    }
  }
  // epilogue: c0,c1 -> pixel m0+g, c2,c3 -> pixel m0+g+8; channels n*8 + 2tg, +1
#pragma unroll
  for (int n = 0; n < NT; n++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int px = m0 + g + 8 * h;
      const size_t p = ((size_t)b * nr + i) * ns + j0 + px;
      const int c = n * 8 + tg * 2;
      float v0 = acc[n][2 * h], v1 = acc[n][2 * h + 1];
      if (MODE == 0) {
        v0 += bias[c];
        v1 += bias[c + 1];
        if (zout) *reinterpret_cast<float2 *>(zout + p * COUT + c) = make_float2(v0, v1);
        *reinterpret_cast<unsigned *>(outb + p * COUT + c) = pack_bf16x2(gelu_f(v0), gelu_f(v1));
      } else if (MODE == 1) {
        *reinterpret_cast<float2 *>(outf + p * COUT + c) = make_float2(v0 + bias[c], v1 + bias[c + 1]);
      } else {
        const float2 z = *reinterpret_cast<const float2 *>(zin + p * COUT + c);
        *reinterpret_cast<unsigned *>(outb + p * COUT + c) = pack_bf16x2(v0 * gelu_grad_f(z.x), v1 * gelu_grad_f(z.y));
      }
    }
  }
}

// Weight and bias gradients: gW[o][tap*CIN + c] += sum_p dz[p][o] x[p + off(tap)][c].
// Each CTA walks `per` tiles (a tile = CL_TILE azimuths of one ring of one
// sample) accumulating in registers, then adds its partial sums atomically.
// M = COUT (rows o), N = 9*CIN (columns k), reduction over pixels.
template <int CIN, int COUT>
__global__ void __launch_bounds__(CL_BS) k_conv_wgrad(const bf16 *__restrict__ x, const bf16 *__restrict__ dz,
                                                      float *__restrict__ gw, float *__restrict__ gb, int nr,
                                                      int ns, int ntiles, int per)
{
  constexpr int XP = CL_TILE + 2 + 8;  // padded transposed row (pixels)
  constexpr int DP = CL_TILE + 8;
  __shared__ __align__(16) bf16 xT[3][CIN][XP];
  __shared__ __align__(16) bf16 dzT[COUT][DP];
  constexpr int MT = COUT / 16;           // m16 tiles
  constexpr int NTT = 9 * CIN / 8;        // n8 tiles in total
  constexpr int NTW = (NTT + 3) / 4;      // per warp
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, tg = lane & 3;
  float acc[MT][NTW][4];
#pragma unroll
  for (int m = 0; m < MT; m++)
#pragma unroll
    for (int n = 0; n < NTW; n++) acc[m][n][0] = acc[m][n][1] = acc[m][n][2] = acc[m][n][3] = 0.f;
  float bsum = 0.f;  // bias gradient of channel tid (tid < COUT)
  const int tiles_per_ring = ns / CL_TILE;
  for (int q = 0; q < per; q++) {
    const int tile = blockIdx.x * per + q;
    if (tile >= ntiles) break;
    const int jt = tile % tiles_per_ring, i = (tile / tiles_per_ring) % nr, b = tile / (tiles_per_ring * nr);
    const int j0 = jt * CL_TILE;
    __syncthreads();  // previous tile's fragments consumed
    for (int t = tid; t < 3 * (CL_TILE + 2) * CIN; t += CL_BS) {
      const int c = t % CIN, px = (t / CIN) % (CL_TILE + 2), r = t / (CIN * (CL_TILE + 2));
      const int ii = i - 1 + r;
      int jj = j0 - 1 + px;
      jj = jj < 0 ? jj + ns : (jj >= ns ? jj - ns : jj);
      xT[r][c][px] = (ii >= 0 && ii < nr) ? x[(((size_t)b * nr + ii) * ns + jj) * CIN + c] : __float2bfloat16(0.f);
    }
    for (int t = tid; t < CL_TILE * COUT; t += CL_BS) {
      const int o = t % COUT, px = t / COUT;
      dzT[o][px] = dz[(((size_t)b * nr + i) * ns + j0 + px) * COUT + o];
    }
    __syncthreads();
    if (tid < COUT) {
      float s = 0.f;
      for (int px = 0; px < CL_TILE; px++) s += __bfloat162float(dzT[tid][px]);
      bsum += s;
    }
#pragma unroll
    for (int kk = 0; kk < CL_TILE / 16; kk++) {
      unsigned a[MT][4];
#pragma unroll
      for (int m = 0; m < MT; m++) {
        a[m][0] = *reinterpret_cast<const unsigned *>(&dzT[m * 16 + g][kk * 16 + tg * 2]);
        a[m][1] = *reinterpret_cast<const unsigned *>(&dzT[m * 16 + g + 8][kk * 16 + tg * 2]);
        a[m][2] = *reinterpret_cast<const unsigned *>(&dzT[m * 16 + g][kk * 16 + 8 + tg * 2]);
        a[m][3] = *reinterpret_cast<const unsigned *>(&dzT[m * 16 + g + 8][kk * 16 + 8 + tg * 2]);
      }
#pragma unroll
      for (int n = 0; n < NTW; n++) {
        const int nt = warp * NTW + n;
        if (nt < NTT) {
          const int col = nt * 8 + g;            // k = tap*CIN + c
          const int tap = col / CIN, c = col % CIN;
          const int dy = tap / 3, dx = tap % 3;
          const int p0 = kk * 16 + tg * 2 + dx;  // halo column of pixel kk*16 + 2tg
          const bf16 *row = &xT[dy][c][0];
          unsigned bb[2];
          {
            __nv_bfloat162 v0, v1;
            v0.x = row[p0]; v0.y = row[p0 + 1];
            v1.x = row[p0 + 8]; v1.y = row[p0 + 9];
            bb[0] = *reinterpret_cast<const unsigned *>(&v0);
            bb[1] = *reinterpret_cast<const unsigned *>(&v1);
          }
#pragma unroll
          for (int m = 0; m < MT; m++) mma_bf16(acc[m][n], a[m], bb);
        }
      }
    }
  }
  // partial sums -> global (rows o = m*16 + g (+8), columns nt*8 + 2tg (+1))
#pragma unroll
  for (int m = 0; m < MT; m++)
#pragma unroll
    for (int n = 0; n < NTW; n++) {
      const int nt = warp * NTW + n;
      if (nt < NTT) {
        const int col = nt * 8 + tg * 2;
        const int o = m * 16 + g;
        atomicAdd(gw + (size_t)o * 9 * CIN + col, acc[m][n][0]);
        atomicAdd(gw + (size_t)o * 9 * CIN + col + 1, acc[m][n][1]);
        atomicAdd(gw + (size_t)(o + 8) * 9 * CIN + col, acc[m][n][2]);
        atomicAdd(gw + (size_t)(o + 8) * 9 * CIN + col + 1, acc[m][n][3]);
      }
    }
  if (tid < COUT) atomicAdd(gb + tid, bsum);
}

// ------------------------------------------------------------ features
// The network's inputs from a coarse disc (FP64 state -> BF16):
//   0: Sigma / SigmaMed(r) - 1          1: vrad / cs(r)
//   2: (vtheta - VthetaMed(r)) / cs(r)  3: (log r - mean) / half-width of log r
//   4: planets' smoothed potential / cs(r)^2 at their current positions
//   5: log10(alpha) + 3                 6: (aspect ratio - 0.065) / 0.035
__global__ void k_features(KP k, bf16 *out, double lmid, double lhalf)
{
  const int i = blockIdx.y, ns = k.ns;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j;
  const double cs = k.cs_ring[i], r = k.rmed[i];
  const fb_ctl *c = k.ctl;
  double phi = 0.0;
  for (int p = 0; p < c->np; p++) {
    const double dx = r * k.cosaz[j] - c->px[p], dy = r * k.sinaz[j] - c->py[p];
    phi -= c->pm[p] / sqrt(dx * dx + dy * dy + c->pot_smooth2[p]);
  }
  float f[CL_CIN];
#pragma unroll
  for (int c = 0; c < CL_CIN; c++) f[c] = 0.f;
  f[0] = (float)(k.rho[l] / k.sigmamed[i] - 1.0);
  f[1] = (float)(k.vr[l] / cs);
  f[2] = (float)((k.vt[l] - k.vthetamed[i]) / cs);
  f[3] = (float)((log(r) - lmid) / lhalf);
  f[4] = (float)(phi / (cs * cs));
  f[5] = (float)(k.alpha > 0.0 ? log10(k.alpha) + 3.0 : -2.0);  // log10 alpha, about -1..1
  f[6] = (float)((k.aspectratio - 0.065) / 0.035);               // h, about -1..1
  unsigned *o = reinterpret_cast<unsigned *>(out + l * CL_CIN);
#pragma unroll
  for (int c = 0; c < CL_CIN; c += 2) o[c / 2] = pack_bf16x2(f[c], f[c + 1]);
}

// Conservative quantities m, J, P of a coarse disc (layout [3][nr][ns]):
// out = sign * U (+ out if accumulate)
__global__ void k_conservative(KP k, float *out, float sign, int accumulate)
{
  const int i = blockIdx.y, ns = k.ns, nr = k.nr;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j, n = (size_t)nr * ns;
  const size_t ljm = (j == 0) ? (size_t)i * ns + ns - 1 : l - 1;
  const double m = k.rho[l];
  const double J = 0.5 * (k.rho[ljm] + k.rho[l]) * k.rmed[i] * k.vt[l];
  const double P = (i >= 1) ? 0.5 * (k.rho[l - ns] + k.rho[l]) * k.vr[l] : 0.0;
  const float u[3] = {(float)m, (float)J, (float)P};
  for (int q = 0; q < 3; q++) {
    float v = sign * u[q];
    if (accumulate) v += out[q * n + l];
    out[q * n + l] = v;
  }
}

// ------------------------------------------------------------ flux differences
// interior radial faces 1..nr-1
static __device__ __forceinline__ int mask_r(int i, int nr) { return (i >= 1 && i <= nr - 1) ? 1 : 0; }
// Sigma0 at radial face i (between rings i-1 and i)
template <typename T>
static __device__ __forceinline__ T sig_face(const T *sig, int i) { return sqrt(sig[i - 1] * sig[i]); }

// dSigma at (i,j) from the network output O (NHWC f32, one sample)
template <typename T, typename S>
static __device__ __forceinline__ T mass_diff(const float *O, T scale, const T *surf, const S *sig, int i, int j,
                                              int nr, int ns)
{
  const size_t row = (size_t)i * ns;
  const int jp = (j == ns - 1) ? 0 : j + 1;
  const T fr0 = mask_r(i, nr) ? (T)O[(row + j) * CL_COUT] * (T)sig_face(sig, i) : (T)0;
  const T fr1 = mask_r(i + 1, nr) ? (T)O[(row + ns + j) * CL_COUT] * (T)sig_face(sig, i + 1) : (T)0;
  const T ft = ((T)O[(row + j) * CL_COUT + 1] - (T)O[(row + jp) * CL_COUT + 1]) * (T)sig[i];
  return scale * ((fr0 - fr1) + ft) / surf[i];
}

// Loss of a minibatch: L = w sum_b sum_ij (dSigma_pred - Y_m)^2 / (B nr ns);
// G = dL/d(dSigma_pred).  One thread per cell and sample; partials per CTA.
__global__ void k_loss(const float *O, const float *Y, const float *sig, const int *idx, const float *scale,
                       const float *wq, const float *surf, float *G, double *loss_part, int nr, int ns, int nb)
{
  __shared__ double sh[256];
  const size_t n = (size_t)nr * ns;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (t < n * nb) {
    const int b = (int)(t / n);
    const size_t l = t - (size_t)b * n;
    const int i = (int)(l / ns), j = (int)(l - (size_t)i * ns);
    const float *Ob = O + (size_t)b * n * CL_COUT;
    const float *Yb = Y + (size_t)idx[b] * 3 * n;
    const float *sb = sig + (size_t)idx[b] * nr;
    const float norm = 1.0f / (float)(n * nb);
    const float d = mass_diff<float, float>(Ob, scale[0], surf, sb, i, j, nr, ns) - Yb[l];
    e = (double)wq[0] * d * d;
    G[(size_t)b * n + l] = 2.0f * wq[0] * d * norm;
  }
  sh[threadIdx.x] = e;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = sh[0] / (double)(n * nb);
}

// dL/dO from G (adjoint of mass_diff); channels >= 2 get 0.  Output bf16
// (the last layer's pre-activation gradient).
__global__ void k_loss_adjoint(const float *G, const float *sig, const int *idx, const float *scale,
                               const float *surf, bf16 *dO, int nr, int ns, int nb)
{
  const size_t n = (size_t)nr * ns;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nb) return;
  const int b = (int)(t / n);
  const size_t l = t - (size_t)b * n;
  const int i = (int)(l / ns), j = (int)(l - (size_t)i * ns);
  const int jm = (j == 0) ? ns - 1 : j - 1;
  const float *Gb = G + (size_t)b * n;
  const float *sb = sig + (size_t)idx[b] * nr;
  const float s = scale[0];
  float d[CL_COUT];
#pragma unroll
  for (int c = 0; c < CL_COUT; c++) d[c] = 0.f;
  // Fr(i,j) enters dSigma(i,j) with +s sf/Surf[i] and dSigma(i-1,j) with -s sf/Surf[i-1]
  if (mask_r(i, nr)) d[0] = s * sig_face(sb, i) * (Gb[l] / surf[i] - Gb[l - ns] / surf[i - 1]);
  // Ft(i,j) enters dSigma(i,j) with +s sig/Surf[i] and dSigma(i,j-1) with -s sig/Surf[i]
  d[1] = s * sb[i] / surf[i] * (Gb[l] - Gb[(size_t)i * ns + jm]);
  unsigned *o = reinterpret_cast<unsigned *>(dO + t * CL_COUT);
#pragma unroll
  for (int c = 0; c < CL_COUT; c += 2) o[c / 2] = pack_bf16x2(d[c], d[c + 1]);
}

// ------------------------------------------------------------ apply (inference)
// At inference each face flux is saturated, F -> Fmax tanh(F/Fmax) with Fmax
// = CL_FMAX in units of the output scale: a pointwise map of the one value
// both cells of a face read, so the correction stays conservative, while an
// output far outside the training range cannot push the disc off.
#define CL_FMAX 3.0
__global__ void k_saturate(const float *O, float *Os, size_t n)
{
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    Os[t] = (float)(CL_FMAX * tanh((double)O[t] / CL_FMAX));
}

// Physical face mass fluxes (FP64) of the saturated outputs: Fr at the
// inner radial face of every cell (ring nr: 0), Ft at its lower azimuthal face.
__global__ void k_face_flux(KP k, const float *O, double scale, double *fr, double *ft)
{
  const int i = blockIdx.y, ns = k.ns, nr = k.nr;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j;
  if (i == nr) {
    fr[l] = 0.0;
    return;
  }
  fr[l] = mask_r(i, nr) ? scale * (double)O[l * CL_COUT] * sig_face(k.sigmamed, i) : 0.0;
  ft[l] = scale * (double)O[l * CL_COUT + 1] * k.sigmamed[i];
}

static __device__ __forceinline__ double dsigma(const KP &k, const double *fr, const double *ft, const double *surf,
                                                int i, int j)
{
  const int ns = k.ns;
  const size_t l = (size_t)i * ns + j;
  const int jp = (j == ns - 1) ? 0 : j + 1;
  return ((fr[l] - fr[l + ns]) + (ft[l] - ft[(size_t)i * ns + jp])) / surf[i];
}

// New density and vtheta (into scratch): mass by the flux differences, the
// angular momentum of every vtheta face's control volume by the same mass
// fluxes carrying the upwind R vtheta.
__global__ void k_apply_mass(KP k, const double *fr, const double *ft, const double *surf, double *rho_new,
                             double *vt_new)
{
  const int i = blockIdx.y, ns = k.ns, nr = k.nr;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const size_t l = (size_t)i * ns + j;
  const int jm = (j == 0) ? ns - 1 : j - 1, jp = (j == ns - 1) ? 0 : j + 1;
  const size_t ljm = (size_t)i * ns + jm, ljp = (size_t)i * ns + jp;
  const double ds = dsigma(k, fr, ft, surf, i, j), dsm = dsigma(k, fr, ft, surf, i, jm);
  const double R = k.rmed[i];
  const double *vt = k.vt;
  // mass through the radial boundaries of the face control volume (i,j)
  const double gin = 0.5 * (fr[ljm] + fr[l]);
  const double gout = 0.5 * (fr[ljm + ns] + fr[l + ns]);
  const double lin = (gin > 0.0) ? k.rmed[i - 1 >= 0 ? i - 1 : 0] * vt[(i >= 1 ? l - ns : l)] : R * vt[l];
  const double lout = (gout > 0.0) ? R * vt[l] : (i + 1 < nr ? k.rmed[i + 1] * vt[l + ns] : R * vt[l]);
  // mass through the cell centres (i,j-1) (in) and (i,j) (out)
  const double tin = 0.5 * (ft[ljm] + ft[l]);
  const double tout = 0.5 * (ft[l] + ft[ljp]);
  const double ltin = (tin > 0.0) ? R * vt[ljm] : R * vt[l];
  const double ltout = (tout > 0.0) ? R * vt[l] : R * vt[ljp];
  const double dJ = ((gin * lin - gout * lout) + (tin * ltin - tout * ltout)) / surf[i];
  const double J = 0.5 * (k.rho[ljm] + k.rho[l]) * R * vt[l] + dJ;
  const double rho_l = k.rho[l] + ds, rho_jm = k.rho[ljm] + dsm;
  rho_new[l] = rho_l;
  vt_new[l] = J / (0.5 * (rho_jm + rho_l) * R);
}

__global__ void k_copy(double *dst, const double *src, size_t n)
{
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    dst[t] = src[t];
}

// ------------------------------------------------------------ downsampling
// Coarse state (factor f in both directions) from a fine one on the same
// radii: Sigma area-weighted, vrad averaged along the coarse radial face,
// vtheta averaged along the coarse azimuthal face.
__global__ void k_downsample(KP fine, KP coarse, int f)
{
  const int I = blockIdx.y, ns = coarse.ns, nsf = fine.ns;
  const int J = blockIdx.x * blockDim.x + threadIdx.x;
  if (J >= ns) return;
  const size_t L = (size_t)I * ns + J;
  double m = 0.0, a = 0.0, vr = 0.0, vt = 0.0;
  for (int p = 0; p < f; p++) {
    const int i = f * I + p;
    double s = 0.0;
    for (int q = 0; q < f; q++) s += fine.rho[(size_t)i * nsf + f * J + q];
    m += fine.surf[i] * s;
    a += fine.surf[i];
    vt += fine.vt[(size_t)i * nsf + f * J];
  }
  for (int q = 0; q < f; q++) vr += fine.vr[(size_t)(f * I) * nsf + f * J + q];
  coarse.rho[L] = m / (a * f);
  coarse.vr[L] = vr / f;
  coarse.vt[L] = vt / f;
}

// ------------------------------------------------------------ optimiser
__global__ void k_adam(float *w, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.f - b1) * gt;
  const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  w[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

// BF16 copies of one layer: forward [o][tap][c], backward [c][8-tap][o]
__global__ void k_pack_weights(const float *w, bf16 *wf, bf16 *wb, int cin, int cout)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cout * 9 * cin) return;
  const int c = t % cin, tap = (t / cin) % 9, o = t / (9 * cin);
  const bf16 v = __float2bfloat16(w[t]);
  wf[t] = v;
  wb[((size_t)c * 9 + (8 - tap)) * cout + o] = v;
}

__global__ void k_stats(const float *Y, const float *sig, const float *surf, int nr, int ns, int count, double *acc)
{
  // acc[0] += Y_m^2, acc[1] += (Y_m Surf / Sigma0)^2
  __shared__ double sh[2][256];
  const size_t n = (size_t)nr * ns;
  double s0 = 0.0, s1 = 0.0;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * count; t += (size_t)gridDim.x * blockDim.x) {
    const size_t smp = t / n, l = t - smp * n;
    const int i = (int)(l / ns);
    const double y = Y[smp * 3 * n + l];
    const double u = y * surf[i] / sig[smp * nr + i];
    s0 += y * y;
    s1 += u * u;
  }
  sh[0][threadIdx.x] = s0;
  sh[1][threadIdx.x] = s1;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomicAdd(acc, sh[0][0]);
    atomicAdd(acc + 1, sh[1][0]);
  }
}

__global__ void k_store_sig(KP k, float *out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < k.nr) out[i] = (float)k.sigmamed[i];
}

// ================================================================== host
struct fb_closure {
  int nr, ns, cap, count;
  cudaStream_t st;
  // per layer: FP32 master weights/biases, BF16 copies, gradients, Adam moments
  float *w[CL_LAYERS], *b[CL_LAYERS], *gw[CL_LAYERS], *gb[CL_LAYERS];
  float *mw[CL_LAYERS], *vw[CL_LAYERS], *mb[CL_LAYERS], *vb[CL_LAYERS];
  bf16 *wf[CL_LAYERS], *wbk[CL_LAYERS];
  int nw[CL_LAYERS];
  int adam_t;
  // output scales and loss weights (float for training, double for apply)
  float *scale_f, *wq_f;
  double *scale_d, *surf_d;
  double *scale_apply;  // scale * gain, used by fb_closure_apply
  double gain;
  float *out_sat;       // saturated outputs (inference)
  float *surf_f;
  float h_scale[3], h_wq[3];
  // dataset
  bf16 *X;
  float *Y;
  float *sig;  // initial density profile of each sample's disc [cap][nr]
  // minibatch work buffers (bmax samples)
  int bmax;
  bf16 *act[CL_LAYERS];   // act[l] = output of layer l (bf16), l < 3
  float *z[CL_LAYERS];    // pre-activations of layers 0..2
  float *out;             // last layer output f32
  bf16 *dz[CL_LAYERS];    // gradient w.r.t. each layer's pre-activation
  float *G;               // dL/d(dq)
  double *loss_part;
  int *idx;
  double *stats;
  // inference scratch
  bf16 *xin;
  double *rho_new, *fr, *ft, *vt_new;
  double lmid, lhalf;
  char err[256];
};

static int cl_alloc(void **p, size_t bytes)
{
  if (cudaMalloc(p, bytes) != cudaSuccess) return FB_ERR_NOMEM;
  cudaMemset(*p, 0, bytes);
  return FB_OK;
}

static unsigned long long cl_rng_next(unsigned long long *s)
{
  // splitmix64
  unsigned long long z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static double cl_gauss(unsigned long long *s)
{
  // Box-Muller on two uniforms in (0,1)
  const double u1 = ((cl_rng_next(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  const double u2 = ((cl_rng_next(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

static void cl_pack(fb_closure *c)
{
  for (int l = 0; l < CL_LAYERS; l++)
    k_pack_weights<<<(c->nw[l] + 255) / 256, 256, 0, c->st>>>(c->w[l], c->wf[l], c->wbk[l], kLayerIn[l], kLayerOut[l]);
}

extern "C" int fb_closure_destroy(fb_closure *c);

extern "C" int fb_closure_create(const fb_ctx *coarse, int capacity, int batch, unsigned long long seed,
                                 fb_closure **out)
{
  if (!coarse || !out || capacity < 1 || batch < 1) return FB_ERR_INVALID;
  *out = NULL;
  const fb_geom *g = fb_ctx_geom(coarse);
  if (!g) return FB_ERR_INVALID;
  if (g->ns % CL_TILE != 0 || g->nr < 3) return FB_ERR_UNSUPPORTED;
  fb_closure *c = new fb_closure();
  memset(c, 0, sizeof *c);
  c->nr = g->nr;
  c->ns = g->ns;
  c->cap = capacity;
  c->bmax = batch;
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) { delete c; return FB_ERR_CUDA; }
  const size_t n = (size_t)c->nr * c->ns;
  int rc = FB_OK;
  unsigned long long s = seed;
  for (int l = 0; l < CL_LAYERS && !rc; l++) {
    const int cin = kLayerIn[l], cout = kLayerOut[l], nw = cout * 9 * cin;
    c->nw[l] = nw;
    // He initialisation over the used input channels; the last layer small,
    // so that training starts near "no correction"
    const int cin_used = (l == 0) ? 7 : cin;
    const double sd = sqrt(2.0 / (9.0 * cin_used)) * (l == CL_LAYERS - 1 ? 0.05 : 1.0);
    std::vector<float> hw(nw);
    for (int t = 0; t < nw; t++) {
      const int ci = t % cin, o = t / (9 * cin);
      const bool used = (ci < cin_used) && (l < CL_LAYERS - 1 || o < 2);
      hw[t] = used ? (float)(sd * cl_gauss(&s)) : 0.0f;
    }
    rc |= cl_alloc((void **)&c->w[l], nw * 4) | cl_alloc((void **)&c->b[l], cout * 4);
    rc |= cl_alloc((void **)&c->gw[l], nw * 4) | cl_alloc((void **)&c->gb[l], cout * 4);
    rc |= cl_alloc((void **)&c->mw[l], nw * 4) | cl_alloc((void **)&c->vw[l], nw * 4);
    rc |= cl_alloc((void **)&c->mb[l], cout * 4) | cl_alloc((void **)&c->vb[l], cout * 4);
    rc |= cl_alloc((void **)&c->wf[l], nw * 2) | cl_alloc((void **)&c->wbk[l], nw * 2);
    if (!rc) cudaMemcpy(c->w[l], hw.data(), nw * 4, cudaMemcpyHostToDevice);
  }
  rc |= cl_alloc((void **)&c->scale_f, 4 * 4) | cl_alloc((void **)&c->wq_f, 4 * 4);
  rc |= cl_alloc((void **)&c->scale_d, 4 * 8) | cl_alloc((void **)&c->surf_d, c->nr * 8);
  rc |= cl_alloc((void **)&c->scale_apply, 4 * 8) | cl_alloc((void **)&c->out_sat, n * CL_COUT * 4);
  rc |= cl_alloc((void **)&c->surf_f, c->nr * 4);
  rc |= cl_alloc((void **)&c->X, (size_t)capacity * n * CL_CIN * 2) | cl_alloc((void **)&c->Y, (size_t)capacity * 3 * n * 4);
  rc |= cl_alloc((void **)&c->sig, (size_t)capacity * c->nr * 4);
  rc |= cl_alloc((void **)&c->fr, (n + c->ns) * 8) | cl_alloc((void **)&c->ft, n * 8) |
        cl_alloc((void **)&c->vt_new, n * 8);
  for (int l = 0; l < CL_LAYERS - 1 && !rc; l++) {
    rc |= cl_alloc((void **)&c->act[l], (size_t)batch * n * CL_C * 2);
    rc |= cl_alloc((void **)&c->z[l], (size_t)batch * n * CL_C * 4);
  }
  rc |= cl_alloc((void **)&c->out, (size_t)batch * n * CL_COUT * 4);
  for (int l = 0; l < CL_LAYERS && !rc; l++) rc |= cl_alloc((void **)&c->dz[l], (size_t)batch * n * kLayerOut[l] * 2);
  rc |= cl_alloc((void **)&c->G, (size_t)batch * 3 * n * 4);
  rc |= cl_alloc((void **)&c->loss_part, ((size_t)batch * n / 256 + 2) * 8);
  rc |= cl_alloc((void **)&c->idx, (size_t)batch * 4) | cl_alloc((void **)&c->stats, 8 * 8);
  rc |= cl_alloc((void **)&c->xin, n * CL_CIN * 2) | cl_alloc((void **)&c->rho_new, (n + c->ns) * 8);
  if (rc) { fb_closure_destroy(c); return FB_ERR_NOMEM; }
  std::vector<double> sd(g->surf, g->surf + c->nr);
  std::vector<float> sf(sd.begin(), sd.end());
  cudaMemcpy(c->surf_d, sd.data(), c->nr * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(c->surf_f, sf.data(), c->nr * 4, cudaMemcpyHostToDevice);
  const double l0 = log(g->rmed[0]), l1 = log(g->rmed[c->nr - 1]);
  c->lmid = 0.5 * (l0 + l1);
  c->lhalf = 0.5 * (l1 - l0);
  for (int q = 0; q < 3; q++) { c->h_scale[q] = 1.0f; c->h_wq[q] = 1.0f; }
  cudaMemcpy(c->scale_f, c->h_scale, 12, cudaMemcpyHostToDevice);
  cudaMemcpy(c->wq_f, c->h_wq, 12, cudaMemcpyHostToDevice);
  double sdd[3] = {1.0, 1.0, 1.0};
  cudaMemcpy(c->scale_d, sdd, 24, cudaMemcpyHostToDevice);
  cudaMemcpy(c->scale_apply, sdd, 24, cudaMemcpyHostToDevice);
  c->gain = 1.0;
  cl_pack(c);
  if (cudaStreamSynchronize(c->st) != cudaSuccess) { fb_closure_destroy(c); return FB_ERR_CUDA; }
  *out = c;
  return FB_OK;
}

extern "C" int fb_closure_destroy(fb_closure *c)
{
  if (!c) return FB_OK;
  if (c->st) cudaStreamSynchronize(c->st);
  for (int l = 0; l < CL_LAYERS; l++) {
    void *p[] = {c->w[l], c->b[l], c->gw[l], c->gb[l], c->mw[l], c->vw[l], c->mb[l], c->vb[l], c->wf[l], c->wbk[l],
                 c->act[l], c->z[l], c->dz[l]};
    for (void *q : p) cudaFree(q);
  }
  void *p[] = {c->scale_f, c->wq_f, c->scale_d, c->scale_apply, c->out_sat, c->surf_d, c->surf_f, c->X, c->Y, c->out, c->G,
               c->loss_part, c->idx, c->stats, c->xin, c->rho_new, c->sig, c->fr, c->ft, c->vt_new};
  for (void *q : p) cudaFree(q);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return FB_OK;
}

extern "C" int fb_closure_num_params(const fb_closure *c, int *nweights, int *nbiases)
{
  if (!c) return FB_ERR_INVALID;
  int a = 0, b = 0;
  for (int l = 0; l < CL_LAYERS; l++) { a += c->nw[l]; b += kLayerOut[l]; }
  if (nweights) *nweights = a;
  if (nbiases) *nbiases = b;
  return FB_OK;
}

// get = 1: copy weights/biases (layer after layer, [o][tap][c]) to host;
// get = 0: set them from host (and refresh the BF16 copies).
extern "C" int fb_closure_params(fb_closure *c, float *w, float *b, int get)
{
  if (!c || !w || !b) return FB_ERR_INVALID;
  size_t ow = 0, ob = 0;
  for (int l = 0; l < CL_LAYERS; l++) {
    const int cout = kLayerOut[l];
    if (get) {
      if (cudaMemcpy(w + ow, c->w[l], c->nw[l] * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return FB_ERR_CUDA;
      if (cudaMemcpy(b + ob, c->b[l], cout * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return FB_ERR_CUDA;
    } else {
      if (cudaMemcpy(c->w[l], w + ow, c->nw[l] * 4, cudaMemcpyHostToDevice) != cudaSuccess) return FB_ERR_CUDA;
      if (cudaMemcpy(c->b[l], b + ob, cout * 4, cudaMemcpyHostToDevice) != cudaSuccess) return FB_ERR_CUDA;
    }
    ow += c->nw[l];
    ob += cout;
  }
  if (!get) {
    cl_pack(c);
    if (cudaStreamSynchronize(c->st) != cudaSuccess) return FB_ERR_CUDA;
  }
  return FB_OK;
}

// scales: 3 output scales (flux units) and 3 loss weights
extern "C" int fb_closure_scales(fb_closure *c, double *scale, double *wq, int get)
{
  if (!c || !scale || !wq) return FB_ERR_INVALID;
  if (get) {
    for (int q = 0; q < 3; q++) { scale[q] = c->h_scale[q]; wq[q] = c->h_wq[q]; }
    return FB_OK;
  }
  for (int q = 0; q < 3; q++) {
    if (!(scale[q] > 0.0) || !(wq[q] > 0.0)) return FB_ERR_INVALID;
    c->h_scale[q] = (float)scale[q];
    c->h_wq[q] = (float)wq[q];
  }
  cudaMemcpy(c->scale_f, c->h_scale, 12, cudaMemcpyHostToDevice);
  cudaMemcpy(c->wq_f, c->h_wq, 12, cudaMemcpyHostToDevice);
  cudaMemcpy(c->scale_d, scale, 24, cudaMemcpyHostToDevice);
  double sa[3] = {scale[0] * c->gain, scale[1] * c->gain, scale[2] * c->gain};
  cudaMemcpy(c->scale_apply, sa, 24, cudaMemcpyHostToDevice);
  return FB_OK;
}

// Strength of the applied correction (1 = as trained); training is unaffected.
extern "C" int fb_closure_set_gain(fb_closure *c, double gain)
{
  if (!c || !(gain >= 0.0) || gain > 10.0) return FB_ERR_INVALID;
  c->gain = gain;
  double sa[3] = {c->h_scale[0] * gain, c->h_scale[1] * gain, c->h_scale[2] * gain};
  return cudaMemcpy(c->scale_apply, sa, 24, cudaMemcpyHostToDevice) == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// Scale and loss weight of the mass correction from the first `count`
// samples: scale = rms(Y_m Surf / Sigma0) (the network's fluxes are then
// O(1)), w = 1 / mean(Y_m^2).  The momentum entries are kept at 1.
extern "C" int fb_closure_autoscale(fb_closure *c, int count)
{
  if (!c || count < 1 || count > c->count) return FB_ERR_INVALID;
  cudaMemsetAsync(c->stats, 0, 8 * 8, c->st);
  k_stats<<<148 * 4, 256, 0, c->st>>>(c->Y, c->sig, c->surf_f, c->nr, c->ns, count, c->stats);
  double h[2];
  if (cudaMemcpyAsync(h, c->stats, 16, cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
      cudaStreamSynchronize(c->st) != cudaSuccess)
    return FB_ERR_CUDA;
  const double n = (double)c->nr * c->ns * count;
  double scale[3] = {1.0, 1.0, 1.0}, wq[3] = {1.0, 1.0, 1.0};
  scale[0] = h[1] > 0.0 ? sqrt(h[1] / n) : 1.0;
  wq[0] = h[0] > 0.0 ? n / h[0] : 1.0;
  return fb_closure_scales(c, scale, wq, 0);
}

static void cl_features(fb_closure *c, const fb_ctx *coarse, bf16 *dst, cudaStream_t s)
{
  const KP &k = *fb_ctx_kp(coarse);
  dim3 gr((c->ns + 127) / 128, c->nr);
  k_features<<<gr, 128, 0, s>>>(k, dst, c->lmid, c->lhalf);
}

// Records one part of training sample `slot` from the coarse disc:
// 0 input features, 1 the plain-method result (Y = -U), 2 the target (Y += U).
extern "C" int fb_closure_record(fb_closure *c, fb_ctx *coarse, int slot, int what)
{
  if (!c || !coarse || slot < 0 || slot >= c->cap || what < 0 || what > 2) return FB_ERR_INVALID;
  const KP *kp = fb_ctx_kp(coarse);
  if (!kp || kp->nr != c->nr || kp->ns != c->ns) return FB_ERR_INVALID;
  cudaStream_t s = fb_ctx_stream(coarse);
  const size_t n = (size_t)c->nr * c->ns;
  if (what == 0) {
    cl_features(c, coarse, c->X + (size_t)slot * n * CL_CIN, s);
    k_store_sig<<<(c->nr + 127) / 128, 128, 0, s>>>(*kp, c->sig + (size_t)slot * c->nr);
  } else {
    dim3 gr((c->ns + 127) / 128, c->nr);
    k_conservative<<<gr, 128, 0, s>>>(*kp, c->Y + (size_t)slot * 3 * n, what == 1 ? -1.0f : 1.0f, what == 2);
    if (what == 2 && slot + 1 > c->count) c->count = slot + 1;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return FB_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// Host-provided sample (features as floats, rounded to BF16; targets;
// initial density profile of the sample's disc).
extern "C" int fb_closure_set_sample(fb_closure *c, int slot, const float *x, const float *y, const float *sig)
{
  if (!c || !x || !y || !sig || slot < 0 || slot >= c->cap) return FB_ERR_INVALID;
  const size_t n = (size_t)c->nr * c->ns;
  std::vector<bf16> hx(n * CL_CIN);
  for (size_t t = 0; t < hx.size(); t++) hx[t] = __float2bfloat16(x[t]);
  if (cudaMemcpy(c->X + (size_t)slot * n * CL_CIN, hx.data(), hx.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->Y + (size_t)slot * 3 * n, y, 3 * n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->sig + (size_t)slot * c->nr, sig, c->nr * 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return FB_ERR_CUDA;
  if (slot + 1 > c->count) c->count = slot + 1;
  return FB_OK;
}

// forward pass of nb samples whose features start at X (contiguous)
static void cl_forward(fb_closure *c, const bf16 *X, int nb, int train, cudaStream_t s)
{
  const int nr = c->nr, ns = c->ns;
  dim3 gr(ns / CL_TILE, nr, nb);
  k_conv<CL_CIN, CL_C, 0><<<gr, CL_BS, 0, s>>>(X, c->wf[0], c->b[0], NULL, c->act[0], NULL, train ? c->z[0] : NULL, nr, ns);
  k_conv<CL_C, CL_C, 0><<<gr, CL_BS, 0, s>>>(c->act[0], c->wf[1], c->b[1], NULL, c->act[1], NULL, train ? c->z[1] : NULL, nr, ns);
  k_conv<CL_C, CL_C, 0><<<gr, CL_BS, 0, s>>>(c->act[1], c->wf[2], c->b[2], NULL, c->act[2], NULL, train ? c->z[2] : NULL, nr, ns);
  k_conv<CL_C, CL_COUT, 1><<<gr, CL_BS, 0, s>>>(c->act[2], c->wf[3], c->b[3], NULL, NULL, c->out, NULL, nr, ns);
}

// loss and gradients of the samples idx[0..nb) (gathered into the batch)
static int cl_loss_grad(fb_closure *c, const int *hidx, int nb, double *loss)
{
  cudaStream_t s = c->st;
  const int nr = c->nr, ns = c->ns;
  const size_t n = (size_t)nr * ns;
  if (nb > c->bmax) return FB_ERR_INVALID;
  // gather the features of the batch contiguously (dz[0] doubles as no scratch: use act buffers)
  bf16 *xb = NULL;
  bool contiguous = true;
  for (int q = 1; q < nb; q++) contiguous &= (hidx[q] == hidx[0] + q);
  if (contiguous) {
    xb = c->X + (size_t)hidx[0] * n * CL_CIN;
  } else {
    if (cudaMallocAsync((void **)&xb, (size_t)nb * n * CL_CIN * 2, s) != cudaSuccess) return FB_ERR_NOMEM;
    for (int q = 0; q < nb; q++)
      cudaMemcpyAsync(xb + (size_t)q * n * CL_CIN, c->X + (size_t)hidx[q] * n * CL_CIN, n * CL_CIN * 2,
                      cudaMemcpyDeviceToDevice, s);
  }
  cudaMemcpyAsync(c->idx, hidx, nb * 4, cudaMemcpyHostToDevice, s);
  cl_forward(c, xb, nb, 1, s);
  const int nblk = (int)((n * nb + 255) / 256);
  k_loss<<<nblk, 256, 0, s>>>(c->out, c->Y, c->sig, c->idx, c->scale_f, c->wq_f, c->surf_f, c->G, c->loss_part, nr, ns,
                              nb);
  k_loss_adjoint<<<nblk, 256, 0, s>>>(c->G, c->sig, c->idx, c->scale_f, c->surf_f, c->dz[3], nr, ns, nb);
  dim3 gr(ns / CL_TILE, nr, nb);
  // backward data: dz[l-1] = conv^T(dz[l]) * GELU'(z[l-1])
  k_conv<CL_COUT, CL_C, 2><<<gr, CL_BS, 0, s>>>(c->dz[3], c->wbk[3], NULL, c->z[2], c->dz[2], NULL, NULL, nr, ns);
  k_conv<CL_C, CL_C, 2><<<gr, CL_BS, 0, s>>>(c->dz[2], c->wbk[2], NULL, c->z[1], c->dz[1], NULL, NULL, nr, ns);
  k_conv<CL_C, CL_C, 2><<<gr, CL_BS, 0, s>>>(c->dz[1], c->wbk[1], NULL, c->z[0], c->dz[0], NULL, NULL, nr, ns);
  // weight gradients
  for (int l = 0; l < CL_LAYERS; l++) {
    cudaMemsetAsync(c->gw[l], 0, c->nw[l] * 4, s);
    cudaMemsetAsync(c->gb[l], 0, kLayerOut[l] * 4, s);
  }
  const int ntiles = nb * nr * (ns / CL_TILE);
  const int per = (ntiles + 148 * 4 - 1) / (148 * 4);
  const int nbw = (ntiles + per - 1) / per;
  k_conv_wgrad<CL_CIN, CL_C><<<nbw, CL_BS, 0, s>>>(xb, c->dz[0], c->gw[0], c->gb[0], nr, ns, ntiles, per);
  k_conv_wgrad<CL_C, CL_C><<<nbw, CL_BS, 0, s>>>(c->act[0], c->dz[1], c->gw[1], c->gb[1], nr, ns, ntiles, per);
  k_conv_wgrad<CL_C, CL_C><<<nbw, CL_BS, 0, s>>>(c->act[1], c->dz[2], c->gw[2], c->gb[2], nr, ns, ntiles, per);
  k_conv_wgrad<CL_C, CL_COUT><<<nbw, CL_BS, 0, s>>>(c->act[2], c->dz[3], c->gw[3], c->gb[3], nr, ns, ntiles, per);
  if (!contiguous) cudaFreeAsync(xb, s);
  if (loss) {
    std::vector<double> lp(nblk);
    if (cudaMemcpyAsync(lp.data(), c->loss_part, nblk * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return FB_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return FB_ERR_CUDA;
    double L = 0.0;
    for (int q = 0; q < nblk; q++) L += lp[q];
    *loss = L;
  }
  return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// Loss and gradients of samples [first, first+nb) without an update (for
// the gradient check); gw/gb may be NULL.
extern "C" int fb_closure_loss_grad(fb_closure *c, int first, int nb, double *loss, float *gw, float *gb)
{
  if (!c || first < 0 || nb < 1 || first + nb > c->count || nb > c->bmax) return FB_ERR_INVALID;
  std::vector<int> idx(nb);
  for (int q = 0; q < nb; q++) idx[q] = first + q;
  int rc = cl_loss_grad(c, idx.data(), nb, loss);
  if (rc) return rc;
  size_t ow = 0, ob = 0;
  for (int l = 0; l < CL_LAYERS; l++) {
    if (gw && cudaMemcpy(gw + ow, c->gw[l], c->nw[l] * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return FB_ERR_CUDA;
    if (gb && cudaMemcpy(gb + ob, c->gb[l], kLayerOut[l] * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return FB_ERR_CUDA;
    ow += c->nw[l];
    ob += kLayerOut[l];
  }
  return FB_OK;
}

// `iters` Adam steps on random minibatches of `nb` samples drawn from
// [first, first+count) with a seeded generator; loss_out[it] = batch loss.
extern "C" int fb_closure_train(fb_closure *c, int first, int count, int nb, int iters, double lr,
                                unsigned long long seed, double *loss_out)
{
  if (!c || first < 0 || count < 1 || first + count > c->count || nb < 1 || nb > c->bmax || iters < 0)
    return FB_ERR_INVALID;
  unsigned long long s = seed;
  std::vector<int> idx(nb);
  for (int it = 0; it < iters; it++) {
    for (int q = 0; q < nb; q++) idx[q] = first + (int)(cl_rng_next(&s) % (unsigned long long)count);
    double L = 0.0;
    int rc = cl_loss_grad(c, idx.data(), nb, loss_out ? &L : NULL);
    if (rc) return rc;
    if (loss_out) loss_out[it] = L;
    c->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)c->adam_t), c2 = 1.f - powf(b2, (float)c->adam_t);
    for (int l = 0; l < CL_LAYERS; l++) {
      k_adam<<<(c->nw[l] + 255) / 256, 256, 0, c->st>>>(c->w[l], c->gw[l], c->mw[l], c->vw[l], c->nw[l], (float)lr, b1,
                                                          b2, 1e-8f, c1, c2);
      k_adam<<<1, 256, 0, c->st>>>(c->b[l], c->gb[l], c->mb[l], c->vb[l], kLayerOut[l], (float)lr, b1, b2, 1e-8f, c1, c2);
    }
    cl_pack(c);
  }
  if (cudaStreamSynchronize(c->st) != cudaSuccess) return FB_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// Network output (NHWC f32, nr*ns*CL_COUT floats) for sample `slot` or, with
// slot < 0, for the coarse disc's current state.
extern "C" int fb_closure_infer(fb_closure *c, const fb_ctx *coarse, int slot, float *out)
{
  if (!c || !out) return FB_ERR_INVALID;
  const size_t n = (size_t)c->nr * c->ns;
  cudaStream_t s = c->st;
  const bf16 *x;
  if (slot >= 0) {
    if (slot >= c->count) return FB_ERR_INVALID;
    x = c->X + (size_t)slot * n * CL_CIN;
  } else {
    if (!coarse) return FB_ERR_INVALID;
    cudaStream_t cs = fb_ctx_stream(coarse);
    cl_features(c, coarse, c->xin, cs);
    if (cudaStreamSynchronize(cs) != cudaSuccess) return FB_ERR_CUDA;
    x = c->xin;
  }
  cl_forward(c, x, 1, 0, s);
  if (cudaMemcpyAsync(out, c->out, n * CL_COUT * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return FB_ERR_CUDA;
  return FB_OK;
}

// One correction of the coarse disc (after a DT of the plain method): the
// network reads the state and its flux corrections are applied in place.
extern "C" int fb_closure_apply(fb_closure *c, fb_ctx *coarse)
{
  if (!c || !coarse) return FB_ERR_INVALID;
  KP *kp = fb_ctx_kp_mut(coarse);
  if (!kp || kp->nr != c->nr || kp->ns != c->ns) return FB_ERR_INVALID;
  cudaStream_t s = fb_ctx_stream(coarse);
  cl_features(c, coarse, c->xin, s);
  // the network on the disc's stream (weights are only written by training)
  const int nr = c->nr, ns = c->ns;
  dim3 gr(ns / CL_TILE, nr, 1);
  k_conv<CL_CIN, CL_C, 0><<<gr, CL_BS, 0, s>>>(c->xin, c->wf[0], c->b[0], NULL, c->act[0], NULL, NULL, nr, ns);
  k_conv<CL_C, CL_C, 0><<<gr, CL_BS, 0, s>>>(c->act[0], c->wf[1], c->b[1], NULL, c->act[1], NULL, NULL, nr, ns);
  k_conv<CL_C, CL_C, 0><<<gr, CL_BS, 0, s>>>(c->act[1], c->wf[2], c->b[2], NULL, c->act[2], NULL, NULL, nr, ns);
  k_conv<CL_C, CL_COUT, 1><<<gr, CL_BS, 0, s>>>(c->act[2], c->wf[3], c->b[3], NULL, NULL, c->out, NULL, nr, ns);
  k_saturate<<<256, 256, 0, s>>>(c->out, c->out_sat, (size_t)nr * ns * CL_COUT);
  k_face_flux<<<dim3((ns + 127) / 128, nr + 1), 128, 0, s>>>(*kp, c->out_sat, (double)c->h_scale[0] * c->gain, c->fr,
                                                               c->ft);
  k_apply_mass<<<dim3((ns + 127) / 128, nr), 128, 0, s>>>(*kp, c->fr, c->ft, c->surf_d, c->rho_new, c->vt_new);
  k_copy<<<256, 256, 0, s>>>(kp->rho, c->rho_new, (size_t)nr * ns);
  k_copy<<<256, 256, 0, s>>>(kp->vt, c->vt_new, (size_t)nr * ns);
  fb_ctx_count_launches(coarse, 10);
  if (cudaStreamSynchronize(s) != cudaSuccess) return FB_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// Coarse disc := factor-f coarse-graining of the fine disc (same radii and
// azimuthal extent); the scalar state (time, planets) is copied.
extern "C" int fb_downsample(const fb_ctx *fine, fb_ctx *coarse)
{
  if (!fine || !coarse) return FB_ERR_INVALID;
  const KP *kf = fb_ctx_kp(fine);
  KP *kc = fb_ctx_kp_mut(coarse);
  if (!kf || !kc || kf->nr % kc->nr || kf->ns % kc->ns) return FB_ERR_INVALID;
  const int f = kf->nr / kc->nr;
  if (f < 1 || kf->ns != f * kc->ns || kf->energy || kc->energy) return FB_ERR_INVALID;
  cudaStream_t sf = fb_ctx_stream(fine), s = fb_ctx_stream(coarse);
  if (cudaStreamSynchronize(sf) != cudaSuccess) return FB_ERR_CUDA;
  dim3 gr((kc->ns + 127) / 128, kc->nr);
  k_downsample<<<gr, 128, 0, s>>>(*kf, *kc, f);
  if (cudaMemcpyAsync(kc->ctl, kf->ctl, sizeof(fb_ctl), cudaMemcpyDeviceToDevice, s) != cudaSuccess) return FB_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return FB_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}
