// fb_noalloc.cu -- fb_transport_noalloc: the transport stage (the same
// kernels as fb_stage(ctx, FB_STAGE_TRANSPORT, dt)) for callers that must not
// allocate device memory.  There is no counterpart in the reference.
//
// Who needs it: a host code that embeds the step inside another GPU
// application which owns the whole device-memory budget (its own pool or
// allocator), or that runs the call from a latency-critical region where
// cudaMalloc/cudaFree are not acceptable (they may synchronize the device).
// Such a caller passes its own device buffers for the fields and gets no
// hidden allocation.
//
// The scratch the transport kernels need between their radial and azimuthal
// passes (six transported quantities and the post-transport density, one
// field each, plus one ring of outflow fluxes) lives in a file-scope
// __device__ array of fixed size (about 7.4 MB): a GPU holds it from the
// first call on it (when the driver loads this file's module) until the
// process exits.  The first call on a device also loads every transport
// kernel, so it is the only call that may make the driver allocate; later
// calls allocate nothing.  A call copies the grid tables from pageable host
// memory and synchronizes its stream, so it must never be made while that
// stream is being captured into a CUDA graph.  Calls share that array and it
// keeps the last call's contents; the only value that must start at zero
// (the outflow accumulator) is cleared on every call.  Calls that overlap on
// the GPU (different streams, or different host threads) race on the shared
// scratch and must be serialised by the caller.
#include <cuda_runtime.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <string.h>
#include "fb_dev.cuh"

#define FB_NA_MAX_CELLS 131072   // (nrad+1)*nsec limit, = FB_NOALLOC_MAX_CELLS
#define FB_NA_MAX_NRAD 4096
#define FB_NA_MAX_NSEC 3072
#define FB_NA_NTAB 10
#define FB_NA_MAX_DEVICES 64
#define FB_NA_MIN_NSEC 16

static __device__ __align__(256) double fb_na_scratch[7 * (size_t)FB_NA_MAX_CELLS + FB_NA_MAX_NSEC];
static __device__ __align__(256) double fb_na_tables[FB_NA_NTAB * (FB_NA_MAX_NRAD + 1)];
static __device__ __align__(256) fb_ctl fb_na_ctl;

struct na_device {
  int ready;
  double *scratch;   // device addresses of the arrays above (cudaGetSymbolAddress)
  double *tables;
  fb_ctl *ctl;
  int smem_ns[2];    // largest nsec the azimuthal kernel attributes were set for
};

static na_device g_na[FB_NA_MAX_DEVICES];
static pthread_mutex_t g_na_lock = PTHREAD_MUTEX_INITIALIZER;
static double g_na_htab[FB_NA_NTAB * (FB_NA_MAX_NRAD + 1)];
static __thread char g_na_err[256];

extern "C" const char *fb_noalloc_last_error(void) { return g_na_err; }

static int na_fail(int code, const char *msg)
{
  snprintf(g_na_err, sizeof g_na_err, "%s", msg);
  return code;
}

// Once per device, with that device current: device addresses of the
// file-scope arrays (host code must not use the symbols themselves), and
// every kernel a call can launch loaded now.  Under lazy module loading
// (CUDA's default) the driver loads a kernel, and may allocate device memory
// for it, the first time the kernel is used; doing all of that here confines
// it to the first call on each device.
static int na_setup(int dev)
{
  na_device &d = g_na[dev];
  if (d.ready) return FB_OK;
  if (cudaGetSymbolAddress((void **)&d.scratch, fb_na_scratch) != cudaSuccess ||
      cudaGetSymbolAddress((void **)&d.tables, fb_na_tables) != cudaSuccess ||
      cudaGetSymbolAddress((void **)&d.ctl, fb_na_ctl) != cudaSuccess) {
    cudaGetLastError();
    return na_fail(FB_ERR_CUDA, "cudaGetSymbolAddress failed for the no-alloc scratch");
  }
  // the azimuthal variants (all of them, whatever the grid) and the radial
  // and vr passes
  if (fb_gas_prepare(FB_NA_MIN_NSEC, 1) != FB_OK || fb_transport_preload() != FB_OK) {
    cudaGetLastError();
    return na_fail(FB_ERR_CUDA, "loading the transport kernels failed");
  }
  d.ready = 1;
  return FB_OK;
}

extern "C" int fb_transport_noalloc(const fb_params *p, double *dens, double *vrad, double *vtheta,
                                    double *energy, double dt, void *stream, double *lost_mass)
{
  if (!p || !dens || !vrad || !vtheta || (p->energy_equation && !energy))
    return na_fail(FB_ERR_INVALID, "null argument");
  if (!(dt > 0.0)) return na_fail(FB_ERR_INVALID, "dt must be > 0");
  const int nr = p->nrad, ns = p->nsec;
  if (nr < 4 || ns < FB_NA_MIN_NSEC) return na_fail(FB_ERR_INVALID, "grid too small (nrad >= 4, nsec >= 16)");
  if ((size_t)(nr + 1) * ns > FB_NA_MAX_CELLS || nr > FB_NA_MAX_NRAD || ns > FB_NA_MAX_NSEC)
    return na_fail(FB_ERR_INVALID,
                   "grid too large for the no-alloc scratch: (nrad+1)*nsec must be <= 131072, "
                   "nrad <= 4096 and nsec <= 3072");
  if (p->unsupported) return na_fail(FB_ERR_UNSUPPORTED, "unsupported .par feature");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= FB_NA_MAX_DEVICES)
    return na_fail(FB_ERR_NODEVICE, "no current CUDA device");
  cudaStream_t s = (cudaStream_t)stream;
  pthread_mutex_lock(&g_na_lock);
  int rc = na_setup(dev);
  na_device &d = g_na[dev];
  const int ei = p->energy_equation ? 1 : 0;
  if (rc == FB_OK && d.smem_ns[ei] < ns) {
    rc = fb_gas_prepare(ns, p->energy_equation);
    if (rc == FB_OK) d.smem_ns[ei] = ns;
    else na_fail(rc, "shared-memory attributes for the azimuthal pass could not be set");
  }
  if (rc != FB_OK) {
    pthread_mutex_unlock(&g_na_lock);
    return rc;
  }
  // 1-D geometry of FillPolar1DArrays (src/SourceEuler.c:80-123) into a
  // static host table, then into the static device table.
  const int T = nr + 1;
  double *rinf = g_na_htab, *rsup = rinf + T, *rmed = rsup + T, *surf = rmed + T;
  double *invrmed = surf + T, *invsurf = invrmed + T, *invdiffrmed = invsurf + T;
  double *dxth = invdiffrmed + T, *invdxth = dxth + T, *radii = invdxth + T;
  memset(g_na_htab, 0, sizeof(double) * FB_NA_NTAB * T);
  {
    const double drrsep = (p->rmax - p->rmin) / (double)nr;
    for (int i = 0; i <= nr; i++)
      radii[i] = p->log_grid ? p->rmin * exp((double)i / (double)nr * log(p->rmax / p->rmin))
                             : p->rmin + drrsep * (double)(i);
    for (int i = 0; i < nr; i++) {
      rinf[i] = radii[i];
      rsup[i] = radii[i + 1];
      rmed[i] = 2.0 / 3.0 * (rsup[i] * rsup[i] * rsup[i] - rinf[i] * rinf[i] * rinf[i]);
      rmed[i] = rmed[i] / (rsup[i] * rsup[i] - rinf[i] * rinf[i]);
      surf[i] = 0.5 * (p->pmax - p->pmin) * (rsup[i] * rsup[i] - rinf[i] * rinf[i]) / (double)ns;
      invrmed[i] = 1.0 / rmed[i];
      invsurf[i] = 1.0 / surf[i];
      dxth[i] = (p->pmax - p->pmin) / (double)ns * rmed[i];
      invdxth[i] = 1.0 / dxth[i];
    }
    rinf[nr] = radii[nr];
    for (int i = 1; i < nr; i++) invdiffrmed[i] = 1.0 / (rmed[i] - rmed[i - 1]);
  }
  cudaError_t e = cudaMemcpyAsync(d.tables, g_na_htab, sizeof(double) * FB_NA_NTAB * T,
                                  cudaMemcpyHostToDevice, s);
  // the outflow accumulator is the only scratch value read before written
  if (e == cudaSuccess) e = cudaMemsetAsync(&d.ctl->lost_mass, 0, sizeof(double), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host table is reused by the next call
  pthread_mutex_unlock(&g_na_lock);
  if (e != cudaSuccess) return na_fail(FB_ERR_CUDA, cudaGetErrorString(e));

  KP k;
  memset(&k, 0, sizeof k);
  k.nr = nr;
  k.ns = ns;
  k.nf = (size_t)(nr + 1) * ns;
  k.cell_bs = 128;
  k.rho = dens;
  k.vr = vrad;
  k.vt = vtheta;
  k.e = energy;
  for (int q = 0; q < 6; q++) k.q[q] = d.scratch + (size_t)q * FB_NA_MAX_CELLS;
  k.rho_t = d.scratch + (size_t)6 * FB_NA_MAX_CELLS;
  k.lost0 = d.scratch + (size_t)7 * FB_NA_MAX_CELLS;
  const double *dt_ = d.tables;
  k.rinf = dt_;
  k.rsup = dt_ + T;
  k.rmed = dt_ + 2 * T;
  k.surf = dt_ + 3 * T;
  k.invrmed = dt_ + 4 * T;
  k.invsurf = dt_ + 5 * T;
  k.invdiffrmed = dt_ + 6 * T;
  k.dxtheta = dt_ + 7 * T;
  k.invdxtheta = dt_ + 8 * T;
  k.ctl = d.ctl;
  k.pmin = p->pmin;
  k.pmax = p->pmax;
  k.omega_frame = p->omegaframe;
  k.energy = p->energy_equation;
  k.fast_transport = p->fast_transport;
  k.transport_only = 1;
  fb_launch_transport(k, dt, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(FB_ERR_CUDA, cudaGetErrorString(e));
  if (lost_mass) {
    e = cudaMemcpyAsync(lost_mass, &d.ctl->lost_mass, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return na_fail(FB_ERR_CUDA, cudaGetErrorString(e));
  }
  return FB_OK;
}
