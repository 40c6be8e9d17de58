// fb_sg.cu -- log-polar self-gravity (sgmain.c, sgkernel.c, sgdens.c,
// sgacc.c, sgupdate.c of the reference) as FP64 FFT kernels for sm_100a.
//
// The reference convolves the reduced densities Sr = Sigma sqrt(r/r0) and
// St = Sr r/r0 with the kernels Kr, Kt on a (2 Nr) x Ns periodic grid (the
// radial direction zero-padded), through unnormalised FFTW transforms:
//     A = IFFT2( -G FFT2(K) . FFT2(S) ),   normalised by rstep tstep/(2Nr Ns).
// Here the transforms are our own, one CTA per 1-D transform or pair:
//   1. sg_rows_fwd : per ring i < Nr, one complex FFT of z = Sr + i St along
//      phi (Stockham, radix 16 in registers first, then 4, 2, 6, 3, 5; lines
//      padded by one slot per 16 in shared memory against bank conflicts;
//      per-pass twiddle tables read with consecutive entries per warp),
//      split into the two half spectra (rows >= Nr are zero, so they are
//      never transformed);
//   2. sg_cols_dif : per pair of azimuthal wavenumbers k and per quantity,
//      the 2 Nr radial points transformed in place (decimation in frequency
//      forward, in time backward, so the spectrum stays in one permuted
//      order in which the kernel spectrum is also stored), product with the
//      kernel spectrum, backward transform; only the Nr physical rows are
//      computed in the last pass and written back (sg_cols, Stockham, for
//      column lengths other than powers of two up to 1024);
//   3. sg_rows_inv : per ring, one inverse complex FFT of Wr + i Wt (both
//      Hermitian), whose real and imaginary parts are the two accelerations,
//      with the normalisation and self-force term of sgacc.c:138-161 fused;
//   4. sg_update   : the velocity kicks of update_sgvelocity (sgupdate.c).
// The kernel spectra are computed once (host glibc for K, device FFT).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>
#include <vector>
#include "fb_dev.cuh"

#define SG_BS 256
#define SG_ROW_BS 128  // threads of a row transform (radix-16 passes: n/16 butterflies)
#define SG_MAXST 16
#define SG_ROW_U 12    // points per thread per load batch of a row (1536 points: one batch)
#define SG_INV_U 8     // wavenumbers per thread per load batch of an inverse row

struct fb_fft_plan {
  int n, nst;
  int radix[SG_MAXST];
  double2 *tw;  // device: exp(-2 pi i t / n), t < n
};

struct FftArgs {
  int n, nst;
  int radix[SG_MAXST];
  const double2 *tw;
};

struct DifArgs {
  int lgm, npass;     // m = 2^lgm; passes of span S_p = m / 16^p >= 32, then the tail
  const double2 *tw;  // pass p: exp(-2 pi i r j / S_p) at [r][j], r < 16, j < S_p / 16
};

struct fb_sg {
  int nr, ns, m, nk;        // m = 2 nr, nk = ns/2 + 1
  fb_fft_plan prow, pcol;
  int p2;                   // 32 <= m = 2^lgm <= 1024: the in-place column kernel
  double2 *tw2;             // its per-pass twiddle tables
  FftArgs frow;             // the row passes (radix 16 first) and their tables
  double2 *twr;
  DifArgs fc2;              // its passes
  double2 *xr, *xt;         // half spectra after the row pass, [i][k], i < nr
  double2 *khr, *kht;       // kernel spectra, [k][m]
  double *sq, *rr;          // sqrt(Rmed/R0), Rmed (per ring) for the densities
  double *nr_accr, *nr_acct;  // per-ring normalisations
  double r0;                // GlobalRmed[0]
  double rstep, tstep, eps;
  size_t smem_row, smem_col, smem_col2;
};

static int plan_radices(int n, int *radix)
{
  int k = 0;
  while (n % 4 == 0 && k < SG_MAXST) { radix[k++] = 4; n /= 4; }
  while (n % 2 == 0 && k < SG_MAXST) { radix[k++] = 2; n /= 2; }
  while (n % 3 == 0 && k < SG_MAXST) { radix[k++] = 3; n /= 3; }
  while (n % 5 == 0 && k < SG_MAXST) { radix[k++] = 5; n /= 5; }
  if (n != 1) return -1;
  return k;
}

static int make_plan(fb_fft_plan *p, int n)
{
  p->n = n;
  p->nst = plan_radices(n, p->radix);
  if (p->nst < 0) return FB_ERR_UNSUPPORTED;
  std::vector<double2> h(n);
  for (int t = 0; t < n; t++) {
    double a = 2.0 * M_PI * (double)t / (double)n;
    h[t] = make_double2(cos(a), -sin(a));
  }
  if (cudaMalloc(&p->tw, n * sizeof(double2)) != cudaSuccess) return FB_ERR_NOMEM;
  cudaMemcpy(p->tw, h.data(), n * sizeof(double2), cudaMemcpyHostToDevice);
  return FB_OK;
}

// Passes of a line of n points, radix 16 first and then 4, 2, 6, 3, 5, with
// their twiddle tables back to back: pass (R, L) holds exp(-2 pi i r jm /
// (L R)) at [r][jm], r < R, jm < L.
static int make_pass_tables(FftArgs *a, double2 **dtab, int n)
{
  a->n = n;
  a->nst = 0;
  int rem = n;
  while (rem % 16 == 0 && a->nst < SG_MAXST) { a->radix[a->nst++] = 16; rem /= 16; }
  int tail[SG_MAXST];
  int nt = plan_radices(rem, tail);
  if (nt < 0 || a->nst + nt > SG_MAXST) return FB_ERR_UNSUPPORTED;
  // a 2 and a 3 make one radix-6 pass instead of two
  int i2 = -1, i3 = -1;
  for (int q = 0; q < nt; q++) {
    if (tail[q] == 2 && i2 < 0) i2 = q;
    if (tail[q] == 3 && i3 < 0) i3 = q;
  }
  if (i2 >= 0 && i3 >= 0) {
    tail[i2] = 6;
    for (int q = i3; q + 1 < nt; q++) tail[q] = tail[q + 1];
    nt--;
  }
  for (int q = 0; q < nt; q++) a->radix[a->nst++] = tail[q];
  for (int q = a->nst; q < SG_MAXST; q++) a->radix[q] = 1;
  std::vector<double2> tab;
  int L = 1;
  for (int st = 0; st < a->nst; st++) {
    const int R = a->radix[st];
    for (int r = 0; r < R; r++)
      for (int jm = 0; jm < L; jm++) {
        const double ang = 2.0 * M_PI * (double)(r * jm) / (double)(L * R);
        tab.push_back(make_double2(cos(ang), -sin(ang)));
      }
    L *= R;
  }
  if (cudaMalloc(dtab, tab.size() * sizeof(double2)) != cudaSuccess) return FB_ERR_NOMEM;
  cudaMemcpy(*dtab, tab.data(), tab.size() * sizeof(double2), cudaMemcpyHostToDevice);
  a->tw = *dtab;
  return FB_OK;
}

// ---------------------------------------------------------------- device FFT
static __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
static __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
static __device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
static __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
static __device__ __forceinline__ double2 crot(double2 a, int inv) { return inv ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x); }


static FftArgs fft_args(const fb_fft_plan &p)
{
  FftArgs a;
  a.n = p.n;
  a.nst = p.nst;
  for (int q = 0; q < SG_MAXST; q++) a.radix[q] = (q < p.nst) ? p.radix[q] : 1;
  a.tw = p.tw;
  return a;
}

// One radix-R pass of a Stockham autosort FFT (all of v[] in registers).
// NL lines of length n lie back to back in x and y.
template <int R, int INV, int NL>
static __device__ __forceinline__ void fft_pass(const double2 *__restrict__ x0, double2 *__restrict__ y0,
                                                int n, int L, const double2 *__restrict__ tw)
{
  const int nr_ = n / R;
  const int tstride = n / (L * R);
  for (int jj = threadIdx.x; jj < NL * nr_; jj += blockDim.x) {
    const int line = (NL == 1) ? 0 : jj / nr_;
    const int j = jj - line * nr_;
    const double2 *__restrict__ x = x0 + (size_t)line * n;
    double2 *__restrict__ y = y0 + (size_t)line * n;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = x[j + r * nr_];
    const int jm = j % L;
    if (L > 1) {
#pragma unroll
      for (int r = 1; r < R; r++) {
        double2 w = tw[r * jm * tstride];  // r*jm*tstride < n
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    if (R == 2) {
      double2 t0 = v[0];
      v[0] = cadd(t0, v[1]);
      v[1] = csub(t0, v[1]);
    } else if (R == 4) {
      double2 A = cadd(v[0], v[2]), B = csub(v[0], v[2]);
      double2 Cc = cadd(v[1], v[3]), D = crot(csub(v[1], v[3]), INV);
      v[0] = cadd(A, Cc);
      v[2] = csub(A, Cc);
      v[1] = cadd(B, D);
      v[3] = csub(B, D);
    } else if (R == 3) {
      const double h = 0.86602540378443864676;  // sqrt(3)/2
      double2 t1 = cadd(v[1], v[2]);
      double2 t2 = csub(v[0], cscale(t1, 0.5));
      double2 t3 = cscale(csub(v[1], v[2]), INV ? h : -h);
      v[0] = cadd(v[0], t1);
      v[1] = make_double2(t2.x - t3.y, t2.y + t3.x);  // t2 + i t3
      v[2] = make_double2(t2.x + t3.y, t2.y - t3.x);  // t2 - i t3
    } else if (R == 5) {  // direct 5-point DFT
      const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
      const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
      const double sg = INV ? 1.0 : -1.0;
      const double cs[5] = {1.0, c1, c2, c2, c1};
      const double sn[5] = {0.0, s1, s2, -s2, -s1};
      double2 in[5];
#pragma unroll
      for (int q = 0; q < 5; q++) in[q] = v[q];
#pragma unroll
      for (int k = 0; k < 5; k++) {
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int q = 0; q < 5; q++) {
          const int e = (k * q) % 5;
          const double c = cs[e], sgn = sg * sn[e];
          re += in[q].x * c - in[q].y * sgn;
          im += in[q].x * sgn + in[q].y * c;
        }
        v[k] = make_double2(re, im);
      }
    }
    const int idxD = (j - jm) * R + jm;
#pragma unroll
    for (int r = 0; r < R; r++) y[idxD + r * L] = v[r];
  }
}

// Stockham autosort FFT of length a.n in shared memory; x holds the input,
// y is scratch; returns the buffer holding the natural-order result.
// inv = 0: sum_j x_j exp(-2 pi i jk/n); inv = 1: exp(+2 pi i jk/n); no scaling.
template <int INV, int NL>
static __device__ double2 *fft_smem_t(double2 *x, double2 *y, const FftArgs &a)
{
  const int n = a.n;
  int L = 1;
  for (int s = 0; s < a.nst; s++) {
    const int R = a.radix[s];
    __syncthreads();
    switch (R) {
      case 4: fft_pass<4, INV, NL>(x, y, n, L, a.tw); break;
      case 2: fft_pass<2, INV, NL>(x, y, n, L, a.tw); break;
      case 3: fft_pass<3, INV, NL>(x, y, n, L, a.tw); break;
      default: fft_pass<5, INV, NL>(x, y, n, L, a.tw); break;
    }
    double2 *t = x;
    x = y;
    y = t;
    L *= R;
  }
  __syncthreads();
  return x;
}


// Radix-R DFT of v[0..R-1] in place (R = 2, 3, 4, 5, 6), natural output order.
template <int R, int INV>
static __device__ __forceinline__ void dft_small(double2 *v);

// 6 = 2 x 3: DFT3 of the even and of the odd points, then
// X[k] = E[k] + w6^k O[k], X[k + 3] = E[k] - w6^k O[k].
template <int INV>
static __device__ __forceinline__ void dft6(double2 *v)
{
  const double h = 0.86602540378443864676;  // sqrt(3)/2
  double2 e[3] = {v[0], v[2], v[4]}, o[3] = {v[1], v[3], v[5]};
  dft_small<3, INV>(e);
  dft_small<3, INV>(o);
  const double2 o1 = cmul(o[1], make_double2(0.5, INV ? h : -h));   // w6
  const double2 o2 = cmul(o[2], make_double2(-0.5, INV ? h : -h));  // w6^2
  v[0] = cadd(e[0], o[0]);
  v[3] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[4] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[5] = csub(e[2], o2);
}

template <int R, int INV>
static __device__ __forceinline__ void dft_small(double2 *v)
{
  if (R == 6) {
    dft6<INV>(v);
  } else if (R == 2) {
    const double2 t0 = v[0];
    v[0] = cadd(t0, v[1]);
    v[1] = csub(t0, v[1]);
  } else if (R == 4) {
    const double2 A = cadd(v[0], v[2]), B = csub(v[0], v[2]);
    const double2 Cc = cadd(v[1], v[3]), D = crot(csub(v[1], v[3]), INV);
    v[0] = cadd(A, Cc);
    v[2] = csub(A, Cc);
    v[1] = cadd(B, D);
    v[3] = csub(B, D);
  } else if (R == 3) {
    const double h = 0.86602540378443864676;  // sqrt(3)/2
    const double2 t1 = cadd(v[1], v[2]);
    const double2 t2 = csub(v[0], cscale(t1, 0.5));
    const double2 t3 = cscale(csub(v[1], v[2]), INV ? h : -h);
    v[0] = cadd(v[0], t1);
    v[1] = make_double2(t2.x - t3.y, t2.y + t3.x);
    v[2] = make_double2(t2.x + t3.y, t2.y - t3.x);
  } else if (R == 5) {
    const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
    const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
    const double sg = INV ? 1.0 : -1.0;
    const double cs[5] = {1.0, c1, c2, c2, c1};
    const double sn[5] = {0.0, s1, s2, -s2, -s1};
    double2 in[5];
#pragma unroll
    for (int q = 0; q < 5; q++) in[q] = v[q];
#pragma unroll
    for (int k = 0; k < 5; k++) {
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int q = 0; q < 5; q++) {
        const int e = (k * q) % 5;
        re += in[q].x * cs[e] - in[q].y * (sg * sn[e]);
        im += in[q].x * (sg * sn[e]) + in[q].y * cs[e];
      }
      v[k] = make_double2(re, im);
    }
  }
}

static __device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }
template <int INV> static __device__ __forceinline__ void dft16(double2 *v);

// v[r] *= w^r (r = 1..15) for a radix-16 pass, w = exp(-/+ 2 pi i jm / (16 L)),
// from the table rows r = 1, 2, 4, 8 alone (tw holds w^r at [r L + jm]); the
// other powers are products of those, at most three deep, a few ulp.  Four
// loads per point instead of fifteen, and fewer registers held.
template <int INV>
static __device__ __forceinline__ void twiddle16(double2 *v, const double2 *__restrict__ tw, int L, int jm)
{
  double2 w1 = tw[L + jm], w2 = tw[2 * L + jm], w4 = tw[4 * L + jm], w8 = tw[8 * L + jm];
  if (INV) { w1.y = -w1.y; w2.y = -w2.y; w4.y = -w4.y; w8.y = -w8.y; }
  const double2 w3 = cmul(w1, w2), w5 = cmul(w4, w1), w6 = cmul(w4, w2), w7 = cmul(w4, w3);
  v[1] = cmul(v[1], w1);
  v[2] = cmul(v[2], w2);
  v[3] = cmul(v[3], w3);
  v[4] = cmul(v[4], w4);
  v[5] = cmul(v[5], w5);
  v[6] = cmul(v[6], w6);
  v[7] = cmul(v[7], w7);
  v[8] = cmul(v[8], w8);
  v[9] = cmul(v[9], cmul(w8, w1));
  v[10] = cmul(v[10], cmul(w8, w2));
  v[11] = cmul(v[11], cmul(w8, w3));
  v[12] = cmul(v[12], cmul(w8, w4));
  v[13] = cmul(v[13], cmul(w8, w5));
  v[14] = cmul(v[14], cmul(w8, w6));
  v[15] = cmul(v[15], cmul(w8, w7));
}

// One radix-R Stockham pass of a line of n points read from a buffer padded
// by one slot per 16; output point p (natural position of this pass) goes
// to out(p, value).  twp is the pass's twiddle table, R rows of L entries
// (exp(-2 pi i r jm / (L R)) at [r][jm], read with consecutive jm per warp).
template <int R, int INV, class Out>
static __device__ __forceinline__ void fft_pass_o(const double2 *__restrict__ x, int n, int L,
                                                  const double2 *__restrict__ twp, Out out)
{
  const int nb = n / R;
  for (int j = threadIdx.x; j < nb; j += blockDim.x) {
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = x[pad16(j + r * nb)];
    const int jm = ((L & (L - 1)) == 0) ? (j & (L - 1)) : (j % L);  // L is a power of two until a 3 or 5
    if (R == 16 && L > 1) {
      twiddle16<INV>(v, twp, L, jm);
    } else if (L > 1) {
#pragma unroll
      for (int r = 1; r < R; r++) {
        double2 w = twp[r * L + jm];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    if (R == 16) dft16<INV>(v); else dft_small<R, INV>(v);
    const int idxD = (j - jm) * R + jm;
#pragma unroll
    for (int r = 0; r < R; r++) out(idxD + r * L, (R == 16) ? v[4 * (r & 3) + (r >> 2)] : v[r]);
  }
}

template <int INV, class Out>
static __device__ __forceinline__ void fft_pass_any(int R, const double2 *x, int n, int L, const double2 *twp, Out out)
{
  switch (R) {
    case 16: fft_pass_o<16, INV>(x, n, L, twp, out); break;
    case 6: fft_pass_o<6, INV>(x, n, L, twp, out); break;
    case 4: fft_pass_o<4, INV>(x, n, L, twp, out); break;
    case 2: fft_pass_o<2, INV>(x, n, L, twp, out); break;
    case 3: fft_pass_o<3, INV>(x, n, L, twp, out); break;
    default: fft_pass_o<5, INV>(x, n, L, twp, out); break;
  }
}

// Stockham FFT of one line in padded shared memory with the passes of a
// (radix 16 first, then 4, 2, 6, 3, 5): the data is in x, y is scratch;
// returns the buffer holding the result.
template <int INV>
static __device__ double2 *fft_line_p(double2 *x, double2 *y, const FftArgs &a)
{
  const int n = a.n;
  int L = 1, off = 0;
  for (int st = 0; st < a.nst; st++) {
    const int R = a.radix[st];
    __syncthreads();
    double2 *yy = y;
    fft_pass_any<INV>(R, x, n, L, a.tw + off, [=](int p, double2 v) { yy[pad16(p)] = v; });
    double2 *t = x;
    x = y;
    y = t;
    off += R * L;
    L *= R;
  }
  __syncthreads();
  return x;
}

// ------------------------------------------------------------------ kernels
// Row pass of compute_fftdensity (sgdens.c:52-68) + the forward transform
// along phi.  in_r/in_t given: real rows are in_r, in_t (kernel setup);
// otherwise Sr, St are built from the density.
__global__ void __launch_bounds__(SG_ROW_BS, 4) sg_rows_fwd(FftArgs fa, int nrows, int ns, int nk,
                                                      const double *dens, const double *sq,
                                                      const double *rmed, double r0,
                                                      const double *in_r, const double *in_t,
                                                      double2 *out_r, double2 *out_t)
{
  fb_grid_dependency();
  extern __shared__ double2 sm[];
  double2 *x = sm, *y = sm + ns + ns / 16;  // padded lines
  const int i = blockIdx.x, T = blockDim.x;
  if (in_r) {
    for (int j = threadIdx.x; j < ns; j += T) x[pad16(j)] = make_double2(in_r[(size_t)i * ns + j], in_t[(size_t)i * ns + j]);
  } else {
    // all of a batch's loads in flight together: one L2 round trip per
    // SG_ROW_U * T points instead of one per T
    const double sqi = sq[i], rmi = rmed[i];
    for (int j0 = 0; j0 < ns; j0 += SG_ROW_U * T) {
      double d[SG_ROW_U];
#pragma unroll
      for (int u = 0; u < SG_ROW_U; u++) {
        const int j = j0 + threadIdx.x + u * T;
        d[u] = (j < ns) ? dens[(size_t)i * ns + j] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < SG_ROW_U; u++) {
        const int j = j0 + threadIdx.x + u * T;
        const double a = d[u] * sqi;   // SGP_Sr = dens*sqrt(Rmed/R0)
        const double b = a * rmi / r0;  // SGP_St = Sr*Rmed/R0
        if (j < ns) x[pad16(j)] = make_double2(a, b);
      }
    }
  }
  double2 *Z = fft_line_p<0>(x, y, fa);
  for (int k = threadIdx.x; k < nk; k += blockDim.x) {
    const double2 zk = Z[pad16(k)], zc = Z[pad16(k ? ns - k : 0)];
    // A = (Z[k] + conj Z[-k]) / 2 ; B = (Z[k] - conj Z[-k]) / (2i)
    const double2 A = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y - zc.y));
    const double2 B = make_double2(0.5 * (zk.y + zc.y), -0.5 * (zk.x - zc.x));
    out_r[(size_t)i * nk + k] = A;
    out_t[(size_t)i * nk + k] = B;
  }
}

// Column pass.  mode 0: forward transform of the kernel half spectra into
// [k][m] layout (setup).  mode 1: forward, product with -G Khat
// (sgacc.c:25-38), inverse, keep rows < nrows_in.
// KC adjacent wavenumbers per CTA: a warp's loads and stores then cover
// whole 32-byte sectors of the [ring][k] spectra (KC*16 bytes per ring)
// instead of half sectors, and the KC transforms share each FFT pass.
#define SG_KC 2
__global__ void __launch_bounds__(SG_BS) sg_cols(FftArgs fa, int nrows_in, int nk, int mode,
                                                  double2 *data_r, double2 *data_t,
                                                  double2 *kh_r, double2 *kh_t)
{
  fb_grid_dependency();
  extern __shared__ double2 sm[];
  const int m = fa.n;
  double2 *x = sm, *y = sm + SG_KC * m;  // SG_KC lines each
  const int k0 = blockIdx.x * SG_KC;
  const int which = blockIdx.y;  // 0: r, 1: t
  double2 *data = which ? data_t : data_r;
  double2 *kh = which ? kh_t : kh_r;
  for (int t = threadIdx.x; t < SG_KC * m; t += blockDim.x) {
    const int i = t / SG_KC, c = t - i * SG_KC, k = k0 + c;
    x[(size_t)c * m + i] = (i < nrows_in && k < nk) ? data[(size_t)i * nk + k] : make_double2(0.0, 0.0);
  }
  // the kernel spectrum of these wavenumbers goes to registers now, so that
  // its loads complete while the forward transform runs
  constexpr int KPT = 8;
  const bool pref = (mode == 1) && (SG_KC * m <= KPT * SG_BS);
  double2 kpre[KPT];
  if (pref) {
#pragma unroll
    for (int q = 0; q < KPT; q++) {
      const int t = threadIdx.x + q * SG_BS;
      const int c = t / m, i = t - c * m, k = k0 + c;
      kpre[q] = (t < SG_KC * m && k < nk) ? kh[(size_t)k * m + i] : make_double2(0.0, 0.0);
    }
  }
  double2 *X = fft_smem_t<0, SG_KC>(x, y, fa);
  if (mode == 0) {
    for (int c = 0; c < SG_KC; c++)
      if (k0 + c < nk)
        for (int i = threadIdx.x; i < m; i += blockDim.x) kh[(size_t)(k0 + c) * m + i] = X[(size_t)c * m + i];
    return;
  }
  if (pref) {
#pragma unroll
    for (int q = 0; q < KPT; q++) {
      const int t = threadIdx.x + q * SG_BS;
      const int c = t / m, k = k0 + c;
      if (t < SG_KC * m && k < nk) {
        const double2 K = kpre[q], S = X[t];
        X[t] = make_double2(-FB_G * (K.x * S.x - K.y * S.y), -FB_G * (K.x * S.y + K.y * S.x));
      }
    }
  } else {
    for (int t = threadIdx.x; t < SG_KC * m; t += blockDim.x) {
      const int c = t / m, i = t - c * m, k = k0 + c;
      if (k < nk) {
        const double2 K = kh[(size_t)k * m + i], S = X[t];
        X[t] = make_double2(-FB_G * (K.x * S.x - K.y * S.y), -FB_G * (K.x * S.y + K.y * S.x));
      }
    }
  }
  double2 *Y = (X == x) ? y : x;
  double2 *W = fft_smem_t<1, SG_KC>(X, Y, fa);
  for (int t = threadIdx.x; t < SG_KC * nrows_in; t += blockDim.x) {
    const int i = t / SG_KC, c = t - i * SG_KC, k = k0 + c;
    if (k < nk) data[(size_t)i * nk + k] = W[(size_t)c * m + i];
  }
}

// ------------------------------------------- column pass, powers of two
// Columns of m = 2^lgm points, 32 <= m <= 1024, transformed in place with
// decimation in frequency forward and decimation in time backward, so that
// no reordering pass is needed: the forward transform leaves the spectrum
// in a fixed permuted order, the kernel spectrum is stored in that same
// order (it is made by the same forward code), the product is pointwise,
// and the backward transform undoes the forward steps in reverse and
// returns natural order.
//   pass p (span S = m / 16^p >= 32): butterflies over the points
//     blk S + j + (S/16) r (r < 16, j < S/16); forward: DFT16, then the
//     outputs times exp(-2 pi i j r' / S); backward: inputs times the
//     conjugate twiddles, then the inverse DFT16;
//   tail (span S <= 16 left): DFTs of S consecutive points, natural order.
// Each thread owns the 16 points of its butterfly (or its 16 consecutive
// points in the tail) for the load and the store of a pass, so a pass
// needs no barrier between them, and nothing is held in registers across
// a barrier: one barrier per pass.  Rows >= m/2 of the input are the zero
// padding (never loaded) and only rows < m/2 of the output are kept (never
// computed past the last butterfly, stored straight to global memory).
// Two adjacent wavenumbers per CTA (thread t: column t & 1, butterfly
// t >> 1): a warp's global loads and stores cover 16 rows x 32 bytes.
// Lines are padded by one slot per 16 and spaced m + m/16 + 4 slots apart,
// which keeps every pass free of bank conflicts.
#define SG_KC2 2

template <int INV>
static __device__ __forceinline__ void dft4(double2 &a, double2 &b, double2 &c, double2 &d)
{
  const double2 A = cadd(a, c), B = csub(a, c);
  const double2 Cc = cadd(b, d), D = crot(csub(b, d), INV);
  a = cadd(A, Cc);
  c = csub(A, Cc);
  b = cadd(B, D);
  d = csub(B, D);
}

// 16-point DFT of v[0..15] in place; output k ends in v[4 (k % 4) + k / 4].
template <int INV>
static __device__ __forceinline__ void dft16(double2 *v)
{
  // exp(-2 pi i e / 16) for e = 1, 2, 3, 6, 9 (e = 4 is -i)
  const double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;
  const double h = 0.70710678118654752440;
  const double sg = INV ? -1.0 : 1.0;  // conjugate for the inverse
#pragma unroll
  for (int s = 0; s < 4; s++) dft4<INV>(v[s], v[s + 4], v[s + 8], v[s + 12]);
  // v[s + 4p] *= W16^(s p)
  v[5] = cmul(v[5], make_double2(c1, -sg * s1));
  v[9] = cmul(v[9], make_double2(h, -sg * h));
  v[13] = cmul(v[13], make_double2(s1, -sg * c1));
  v[6] = cmul(v[6], make_double2(h, -sg * h));
  v[10] = crot(v[10], INV);
  v[14] = cmul(v[14], make_double2(-h, -sg * h));
  v[7] = cmul(v[7], make_double2(s1, -sg * c1));
  v[11] = cmul(v[11], make_double2(-h, -sg * h));
  v[15] = cmul(v[15], make_double2(-c1, sg * s1));
#pragma unroll
  for (int p = 0; p < 4; p++) dft4<INV>(v[4 * p], v[4 * p + 1], v[4 * p + 2], v[4 * p + 3]);
}


// 8-point DFT of v[0..7] in place, natural order (radix 2 x 4).
template <int INV>
static __device__ __forceinline__ void dft8(double2 *v)
{
  const double h = 0.70710678118654752440;
  const double sg = INV ? -1.0 : 1.0;
  double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  o1 = cmul(o1, make_double2(h, -sg * h));
  o2 = crot(o2, INV);
  o3 = cmul(o3, make_double2(-h, -sg * h));
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

// The tail: DFTs of S consecutive points (S = 2, 4, 8, 16) over v[0..15].
template <int INV>
static __device__ __forceinline__ void dif_tail(double2 *v, int S)
{
  if (S == 16) {
    dft16<INV>(v);
    double2 w[16];
#pragma unroll
    for (int r = 0; r < 16; r++) w[r] = v[4 * (r & 3) + (r >> 2)];
#pragma unroll
    for (int r = 0; r < 16; r++) v[r] = w[r];
  } else if (S == 8) {
    dft8<INV>(v);
    dft8<INV>(v + 8);
  } else if (S == 4) {
#pragma unroll
    for (int g = 0; g < 4; g++) dft4<INV>(v[4 * g], v[4 * g + 1], v[4 * g + 2], v[4 * g + 3]);
  } else {
#pragma unroll
    for (int g = 0; g < 8; g++) {
      const double2 t0 = v[2 * g];
      v[2 * g] = cadd(t0, v[2 * g + 1]);
      v[2 * g + 1] = csub(t0, v[2 * g + 1]);
    }
  }
}

// A shared pass of span S over line x (forward: DFT16 then twiddles;
// backward: conjugate twiddles then inverse DFT16).  q < m/16 butterflies.
template <int INV>
static __device__ __forceinline__ void dif_pass(double2 *x, int S, int q, const double2 *__restrict__ tw)
{
  const int sb = S >> 4, j = q & (sb - 1), base = (q - j) * 16 + j;  // blk S + j, blk = q / sb
  double2 v[16];
#pragma unroll
  for (int r = 0; r < 16; r++) v[r] = x[pad16(base + r * sb)];
  if (INV) {
#pragma unroll
    for (int r = 1; r < 16; r++) {
      double2 w = tw[r * sb + j];
      w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
  }
  dft16<INV>(v);
#pragma unroll
  for (int r = 0; r < 16; r++) {
    double2 o = v[4 * (r & 3) + (r >> 2)];
    if (!INV && r > 0) o = cmul(o, tw[r * sb + j]);
    x[pad16(base + r * sb)] = o;
  }
}

// MODE 0: forward transform of full columns (all m rows of data) into kh,
// in the permuted order, the tail point r of thread q at [r][q] (setup of
// the kernel spectra; MODE 1 reads it back the same way).  MODE 1: the
// convolution of compute_sgacc (sgacc.c:25-38): forward transform of the
// zero-padded half spectra, product with -G Khat, backward transform, rows
// < m/2 written back into data.
template <int MODE>
__global__ void __launch_bounds__(128, 4) sg_cols_dif(DifArgs da, int nk, double2 *data_r, double2 *data_t,
                                                  double2 *kh_r, double2 *kh_t)
{
  const int m = 1 << da.lgm, q16 = m >> 4, mp = m + q16 + 4, tid = threadIdx.x;
  const int c = tid & 1, q = tid >> 1, k = blockIdx.x * SG_KC2 + c;
  const bool live = k < nk;
  double2 *data = blockIdx.y ? data_t : data_r;
  double2 *kh = blockIdx.y ? kh_t : kh_r;
  if (MODE == 1 && tid == 0) {
    // this CTA's kernel spectra (constant: no wait on the previous grid)
    // into L2 while the forward transform runs
    const int k0 = blockIdx.x * SG_KC2, nc = (nk - k0 < SG_KC2) ? nk - k0 : SG_KC2;
    const double2 *src = kh + (size_t)k0 * m;
    const unsigned bytes = (unsigned)(nc * m * sizeof(double2));
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
  }
  fb_grid_dependency();
  extern __shared__ double2 sm[];
  double2 *x = sm + c * mp;
  double2 v[16];
  // pass 0 (span m) from global memory: points q + r m/16
#pragma unroll
  for (int r = 0; r < 16; r++)
    v[r] = (live && (MODE == 0 || r < 8)) ? data[(size_t)(q + r * q16) * nk + k] : make_double2(0.0, 0.0);
  dft16<0>(v);
#pragma unroll
  for (int r = 0; r < 16; r++) {
    double2 o = v[4 * (r & 3) + (r >> 2)];
    if (r > 0) o = cmul(o, da.tw[r * q16 + q]);
    x[pad16(q + r * q16)] = o;
  }
  __syncthreads();
  int S = q16, off = m;  // the pass-0 table has 16 (m/16) entries
  for (int p = 1; p < da.npass; p++) {
    dif_pass<0>(x, S, q, da.tw + off);
    __syncthreads();
    off += S;
    S >>= 4;
  }
  // tail: the thread's 16 consecutive points
#pragma unroll
  for (int r = 0; r < 16; r++) v[r] = x[pad16(16 * q + r)];
  dif_tail<0>(v, S);
  if constexpr (MODE == 0) {
    if (live) {
#pragma unroll
      for (int r = 0; r < 16; r++) kh[(size_t)k * m + r * q16 + q] = v[r];  // [r][q]: coalesced
    }
  } else {
#pragma unroll
    for (int r = 0; r < 16; r++) {
      const double2 K = live ? kh[(size_t)k * m + r * q16 + q] : make_double2(0.0, 0.0), Sv = v[r];
      v[r] = make_double2(-FB_G * (K.x * Sv.x - K.y * Sv.y), -FB_G * (K.x * Sv.y + K.y * Sv.x));
    }
    dif_tail<1>(v, S);
#pragma unroll
    for (int r = 0; r < 16; r++) x[pad16(16 * q + r)] = v[r];
    __syncthreads();
    for (int p = da.npass - 1; p >= 1; p--) {
      S <<= 4;
      off -= S;
      dif_pass<1>(x, S, q, da.tw + off);
      __syncthreads();
    }
    // backward pass 0: rows q + r' m/16 for r' < 8 only
#pragma unroll
    for (int r = 0; r < 16; r++) v[r] = x[pad16(q + r * q16)];
#pragma unroll
    for (int r = 1; r < 16; r++) {
      double2 w = da.tw[r * q16 + q];
      w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
    dft16<1>(v);
    if (live) {
#pragma unroll
      for (int r = 0; r < 8; r++) data[(size_t)(q + r * q16) * nk + k] = v[4 * (r & 3) + (r >> 2)];
    }
  }
}

// Inverse row pass + sgacc.c:138-161: normalisation, self-force.
__global__ void __launch_bounds__(SG_ROW_BS, 4) sg_rows_inv(FftArgs fa, int ns, int nk, const double2 *wr,
                                                      const double2 *wt, const double *normr,
                                                      const double *normt, const double *dens,
                                                      double selfk_rstep, double selfk_tstep,
                                                      double eps, double *accr, double *acct)
{
  fb_grid_dependency();
  extern __shared__ double2 sm[];
  double2 *x = sm, *y = sm + ns + ns / 16;  // padded lines
  const int i = blockIdx.x, T = blockDim.x;
  const double nrm_r = normr[i], nrm_t = normt[i];
  const double *di = dens + (size_t)i * ns;
  double *ar_i = accr + (size_t)i * ns, *at_i = acct + (size_t)i * ns;
  // each stored wavenumber k < nk is read once and gives x[k] and, for
  // 0 < k with ns - k >= nk, its Hermitian mirror x[ns - k]
  for (int k0 = 0; k0 < nk; k0 += SG_INV_U * T) {
    double2 a[SG_INV_U], b[SG_INV_U];
#pragma unroll
    for (int u = 0; u < SG_INV_U; u++) {
      const int k = k0 + threadIdx.x + u * T;
      a[u] = (k < nk) ? wr[(size_t)i * nk + k] : make_double2(0.0, 0.0);
      b[u] = (k < nk) ? wt[(size_t)i * nk + k] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < SG_INV_U; u++) {
      const int k = k0 + threadIdx.x + u * T;
      if (k >= nk) continue;
      const double2 p = a[u], q = b[u];
      if (k >= 1 && ns - k >= nk) x[pad16(ns - k)] = make_double2(p.x + q.y, -p.y + q.x);  // conj p + i conj q
      if (k == 0 || 2 * k == ns) x[pad16(k)] = make_double2(p.x, q.x);  // c2r reads only Re there
      else x[pad16(k)] = make_double2(p.x - q.y, p.y + q.x);             // p + i q
    }
  }
  double2 *A = fft_line_p<1>(x, y, fa);
  for (int j0 = 0; j0 < ns; j0 += SG_ROW_U * T) {
    double d[SG_ROW_U];
#pragma unroll
    for (int u = 0; u < SG_ROW_U; u++) {
      const int j = j0 + threadIdx.x + u * T;
      d[u] = (j < ns) ? di[j] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < SG_ROW_U; u++) {
      const int j = j0 + threadIdx.x + u * T;
      if (j >= ns) continue;
      const double2 aj = A[pad16(j)];
      double ar = aj.x * nrm_r;
      ar += FB_G * d[u] * selfk_rstep * selfk_tstep / eps;
      ar_i[j] = ar;
      at_i[j] = aj.y * nrm_t;
    }
  }
}

// update_sgvelocity (sgupdate.c:30-72) on VradInt / VthetaInt.  refresh = 1
// is the call the reference's main loop makes before every DT
// (main.c:316, Dt = 0, on Vrad / Vtheta), which matters only for the
// RadSGAcc / AziSGAcc grids the particles read.
__global__ void __launch_bounds__(SG_BS) sg_update(KP k, int refresh)
{
  fb_grid_dependency();
  const int ns = k.ns;
  const int i = blockIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  const double Dt = refresh ? 0.0 : k.ctl->dt;
  double *vr = refresh ? k.vr : k.vri;
  double *vt = refresh ? k.vt : k.vti;
  const size_t l = (size_t)i * ns + j;
  const size_t lm1 = (size_t)i * ns + (j == 0 ? ns - 1 : j - 1);
  // every load first
  const double at0 = k.sg_acct[l], at1 = k.sg_acct[lm1], vtl = vt[l];
  double ar0 = 0.0, ar1 = 0.0, vrl = 0.0, c0 = 0.0, c1 = 0.0, invd = 0.0;
  if (i > 0) {
    ar0 = k.sg_accr[l];
    ar1 = k.sg_accr[l - ns];
    vrl = vr[l];
    c0 = k.rinf[i] - k.rmed[i - 1];
    c1 = k.rmed[i] - k.rinf[i];
    invd = k.invdiffrmed[i];
  }
  if (i > 0) {
    const double radsgacc = (c0 * ar0 + c1 * ar1) * invd;
    vr[l] = vrl + Dt * radsgacc;
    if (k.particles) k.rsga[l] = radsgacc;
  }
  const double azisgacc = 0.5 * (at0 + at1);
  vt[l] = vtl + Dt * azisgacc;
  if (k.particles) k.asga[l] = azisgacc;
}

// ------------------------------------------------------------------- host
int fb_sg_create(fb_sg **out, const fb_params *p, const fb_geom *g, cudaStream_t s)
{
  *out = NULL;
  fb_sg *sg = new fb_sg();
  memset(sg, 0, sizeof *sg);
  const int nr = g->nr, ns = g->ns, m = 2 * nr, nk = ns / 2 + 1;
  sg->nr = nr;
  sg->ns = ns;
  sg->m = m;
  sg->nk = nk;
  if (ns % 2 != 0) { delete sg; return FB_ERR_UNSUPPORTED; }
  int rc = make_plan(&sg->prow, ns);
  if (!rc) rc = make_plan(&sg->pcol, m);
  if (!rc) rc = make_pass_tables(&sg->frow, &sg->twr, ns);
  if (rc) { fb_sg_destroy(sg); return rc; }
  sg->smem_row = 2 * ((size_t)ns + ns / 16) * sizeof(double2);  // two padded lines
  sg->smem_col = 2 * (size_t)SG_KC * m * sizeof(double2);
  sg->p2 = (m >= 32 && m <= 1024 && (m & (m - 1)) == 0);  // CTAs of 2m/16 <= 128 threads
  if (sg->p2) {
    DifArgs &a = sg->fc2;
    a.lgm = 0;
    while ((1 << a.lgm) < m) a.lgm++;
    // pass tables: exp(-2 pi i r j / S) at [r][j], r < 16, j < S/16, S = m, m/16, ... >= 32
    std::vector<double2> tab;
    a.npass = 0;
    for (int S = m; S >= 32; S /= 16) {
      a.npass++;
      for (int r = 0; r < 16; r++)
        for (int j = 0; j < S / 16; j++) {
          const double ang = 2.0 * M_PI * (double)((r * j) % S) / (double)S;
          tab.push_back(make_double2(cos(ang), -sin(ang)));
        }
    }
    if (cudaMalloc(&sg->tw2, tab.size() * sizeof(double2)) != cudaSuccess) { fb_sg_destroy(sg); return FB_ERR_NOMEM; }
    cudaMemcpy(sg->tw2, tab.data(), tab.size() * sizeof(double2), cudaMemcpyHostToDevice);
    a.tw = sg->tw2;
    sg->smem_col2 = (size_t)SG_KC2 * (m + m / 16 + 4) * sizeof(double2);
  }
  int dev = 0, maxopt = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (sg->smem_row > (size_t)maxopt || sg->smem_col > (size_t)maxopt) { fb_sg_destroy(sg); return FB_ERR_UNSUPPORTED; }
  if (fb_allow_max_dynamic_smem((const void *)sg_rows_fwd) || fb_allow_max_dynamic_smem((const void *)sg_rows_inv) ||
      fb_allow_max_dynamic_smem((const void *)sg_cols) || fb_allow_max_dynamic_smem((const void *)sg_cols_dif<0>) ||
      fb_allow_max_dynamic_smem((const void *)sg_cols_dif<1>)) {
    fb_sg_destroy(sg);
    return FB_ERR_CUDA;
  }
  // init_sg (sginit.c:9-11)
  sg->eps = p->sgthicknesssmoothing * p->aspectratio;
  sg->rstep = log(g->radii[nr] / g->radii[0]) / (double)nr;
  sg->tstep = (p->pmax - p->pmin) / (double)ns;
  // per-ring factors
  std::vector<double> sq(nr), normr(nr), normt(nr);
  const double r0 = g->rmed[0];
  sg->r0 = r0;
  for (int i = 0; i < nr; i++) {
    sq[i] = sqrt(g->rmed[i] / r0);
    double normaccr = sg->rstep * sg->tstep / ((double)(2 * nr) * (double)ns);
    double normacct = normaccr;
    normaccr /= sqrt(g->rmed[i] / r0);
    normacct /= (g->rmed[i] / r0 * sqrt(g->rmed[i] / r0));
    normr[i] = normaccr;
    normt[i] = normacct;
  }
  bool ok = cudaMalloc(&sg->xr, (size_t)nr * nk * sizeof(double2)) == cudaSuccess &&
            cudaMalloc(&sg->xt, (size_t)nr * nk * sizeof(double2)) == cudaSuccess &&
            cudaMalloc(&sg->khr, (size_t)nk * m * sizeof(double2)) == cudaSuccess &&
            cudaMalloc(&sg->kht, (size_t)nk * m * sizeof(double2)) == cudaSuccess &&
            cudaMalloc(&sg->sq, nr * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&sg->rr, nr * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&sg->nr_accr, nr * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&sg->nr_acct, nr * sizeof(double)) == cudaSuccess;
  if (!ok) { fb_sg_destroy(sg); return FB_ERR_NOMEM; }
  cudaMemcpy(sg->sq, sq.data(), nr * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(sg->rr, g->rmed, nr * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(sg->nr_accr, normr.data(), nr * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(sg->nr_acct, normt.data(), nr * sizeof(double), cudaMemcpyHostToDevice);
  // compute_fftkernel (sgkernel.c:3-27): kernels on the 2 Nr x Ns grid
  std::vector<double> kr((size_t)m * ns), kt((size_t)m * ns);
  const double e2 = sg->eps * sg->eps;
  for (int i = 0; i < m; i++) {
    double u;
    if (i < nr)
      u = log(g->radii[i] / g->radii[0]);
    else
      u = -log(g->radii[2 * nr - i] / g->radii[0]);
    for (int j = 0; j < ns; j++) {
      const size_t l = (size_t)i * ns + j;
      double a = 1.0 + sg->eps * sg->eps - g->cosaz[j] * exp(-u);
      a *= pow(sg->eps * sg->eps * exp(u) + 2.0 * (cosh(u) - g->cosaz[j]), -1.5);
      double b = g->sinaz[j];
      b *= pow(sg->eps * sg->eps * exp(u) + 2.0 * (cosh(u) - g->cosaz[j]), -1.5);
      kr[l] = a;
      kt[l] = b;
    }
  }
  (void)e2;
  double *dkr = NULL, *dkt = NULL;
  double2 *hr = NULL, *ht = NULL;
  ok = cudaMalloc(&dkr, kr.size() * sizeof(double)) == cudaSuccess &&
       cudaMalloc(&dkt, kt.size() * sizeof(double)) == cudaSuccess &&
       cudaMalloc(&hr, (size_t)m * nk * sizeof(double2)) == cudaSuccess &&
       cudaMalloc(&ht, (size_t)m * nk * sizeof(double2)) == cudaSuccess;
  if (!ok) { cudaFree(dkr); cudaFree(dkt); cudaFree(hr); cudaFree(ht); fb_sg_destroy(sg); return FB_ERR_NOMEM; }
  cudaMemcpy(dkr, kr.data(), kr.size() * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(dkt, kt.data(), kt.size() * sizeof(double), cudaMemcpyHostToDevice);
  FftArgs fc = fft_args(sg->pcol);
  fb_launch(sg_rows_fwd, m, SG_ROW_BS, sg->smem_row, s, sg->frow, m, ns, nk, nullptr, nullptr, nullptr, 1.0, dkr, dkt, hr, ht);
  if (sg->p2)
    fb_launch(sg_cols_dif<0>, dim3((nk + SG_KC2 - 1) / SG_KC2, 2), SG_KC2 * m / 16, sg->smem_col2, s, sg->fc2, nk, hr, ht,
              sg->khr, sg->kht);
  else
    fb_launch(sg_cols, dim3((nk + SG_KC - 1) / SG_KC, 2), SG_BS, sg->smem_col, s, fc, m, nk, 0, hr, ht, sg->khr, sg->kht);
  cudaError_t e = cudaStreamSynchronize(s);
  cudaFree(dkr); cudaFree(dkt); cudaFree(hr); cudaFree(ht);
  if (e != cudaSuccess) { fb_sg_destroy(sg); return FB_ERR_CUDA; }
  *out = sg;
  return FB_OK;
}

void fb_sg_destroy(fb_sg *sg)
{
  if (!sg) return;
  cudaFree(sg->prow.tw); cudaFree(sg->pcol.tw); cudaFree(sg->tw2); cudaFree(sg->twr);
  cudaFree(sg->xr); cudaFree(sg->xt); cudaFree(sg->khr); cudaFree(sg->kht);
  cudaFree(sg->sq); cudaFree(sg->rr); cudaFree(sg->nr_accr); cudaFree(sg->nr_acct);
  delete sg;
}

// compute_fftdensity + compute_sgacc (sgdens.c, sgacc.c): 3 launches
void fb_sg_rows_fwd(fb_sg *sg, const KP &k, const double *dens, cudaStream_t s)
{
  (void)k;
  fb_launch(sg_rows_fwd, sg->nr, SG_ROW_BS, sg->smem_row, s, sg->frow, sg->nr, sg->ns, sg->nk, dens, sg->sq, sg->rr, sg->r0,
                                                   nullptr, nullptr, sg->xr, sg->xt);
}

void fb_sg_cols(fb_sg *sg, cudaStream_t s)
{
  if (sg->p2) {
    fb_launch(sg_cols_dif<1>, dim3((sg->nk + SG_KC2 - 1) / SG_KC2, 2), SG_KC2 * sg->m / 16, sg->smem_col2, s, sg->fc2,
              sg->nk, sg->xr, sg->xt, sg->khr, sg->kht);
    return;
  }
  FftArgs fc = fft_args(sg->pcol);
  fb_launch(sg_cols, dim3((sg->nk + SG_KC - 1) / SG_KC, 2), SG_BS, sg->smem_col, s, fc, sg->nr, sg->nk, 1, sg->xr, sg->xt,
                                                                         sg->khr, sg->kht);
}

void fb_sg_rows_inv(fb_sg *sg, const KP &k, const double *dens, cudaStream_t s)
{
  fb_launch(sg_rows_inv, sg->nr, SG_ROW_BS, sg->smem_row, s, sg->frow, sg->ns, sg->nk, sg->xr, sg->xt, sg->nr_accr, sg->nr_acct,
                                                   dens, sg->rstep, sg->tstep, sg->eps, k.sg_accr, k.sg_acct);
}

void fb_sg_accel(fb_sg *sg, const KP &k, const double *dens, cudaStream_t s)
{
  fb_sg_rows_fwd(sg, k, dens, s);
  fb_sg_cols(sg, s);
  fb_sg_rows_inv(sg, k, dens, s);
}

void fb_sg_update_velocities(const KP &k, cudaStream_t s, int refresh)
{
  fb_launch(sg_update, dim3((k.ns + SG_BS - 1) / SG_BS, k.nr), SG_BS, 0, s, k, refresh);
}

int fb_sg_launches(const fb_sg *sg) { return sg ? 4 : 0; }

extern "C" int fb_sg_ready(void) { return 1; }
