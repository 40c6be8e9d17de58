/* fb_internal.h -- declarations shared by the C host code (fb_host.c) and the
 * CUDA part (fb_*.cu) of libfargo_b200.so.  Not part of the public ABI. */
#ifndef FB_INTERNAL_H
#define FB_INTERNAL_H

#include "fargo_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Constants of src/fondam.h and src/SourceEuler.c:10-13. */
#define FB_G 1.0
#define FB_PI 3.14159265358979323844
#define FB_CFLSECURITY 0.5
#define FB_CVNR 1.41
#define FB_BINARYSECURITY 100.0

/* Unsupported-feature bits of fb_params.unsupported */
#define FB_U_CENTRIFUGAL      (1ull << 0)
#define FB_U_TAILOFF          (1ull << 1)
#define FB_U_DUSTFLUID        (1ull << 2)
#define FB_U_BOUNDARY         (1ull << 3)
#define FB_U_OUTERSOURCE      (1ull << 4)
#define FB_U_DAMPTOVISCOUS    (1ull << 5)
#define FB_U_ADDMASS          (1ull << 6)
#define FB_U_EVAPORATION      (1ull << 7)
#define FB_U_PHOTOEVAP        (1ull << 8)
#define FB_U_SGZEROMODE       (1ull << 9)
#define FB_U_ZMPLUS           (1ull << 10)
#define FB_U_MHDLSA           (1ull << 11)
#define FB_U_THERMALDIFF      (1ull << 12)
#define FB_U_THERMALCOOLING   (1ull << 13)
#define FB_U_TEMPPRESC        (1ull << 14)
#define FB_U_COROTATING       (1ull << 15)
#define FB_U_CICPLANET        (1ull << 16)
#define FB_U_BM08             (1ull << 17)
#define FB_U_CPDMASS          (1ull << 18)
#define FB_U_LABEL            (1ull << 19)
#define FB_U_IMPOSEDDENSITY   (1ull << 20)
#define FB_U_ADDM             (1ull << 21)
#define FB_U_CAVITY           (1ull << 22)
#define FB_U_TRANSITION       (1ull << 23)
#define FB_U_LAMBDADOUBLING   (1ull << 24)
#define FB_U_RELEASE          (1ull << 25)
#define FB_U_FORCEDINNER      (1ull << 26)
#define FB_U_RADIIFILE        (1ull << 27)
#define FB_U_VISCRELEASE      (1ull << 28)
#define FB_U_DUSTTIMESTEP     (1ull << 29)
#define FB_U_PARTICLES        (1ull << 30)
#define FB_U_ADDNOISE         (1ull << 31)
#define FB_U_PLANETACCRETION  (1ull << 32)
#define FB_U_FEELDISK         (1ull << 33)
#define FB_U_BINARY           (1ull << 34)
#define FB_U_FEELOTHERS_FC    (1ull << 35)
#define FB_U_ZZINTEGRATOR     (1ull << 37)
#define FB_U_DUSTGROWTH       (1ull << 38)
#define FB_U_HILLREMOVAL      (1ull << 39)
#define FB_U_INTERPOLATION    (1ull << 40)
#define FB_U_DUSTSGZERO       (1ull << 41)
#define FB_U_SOFTWRITING      (1ull << 42)
#define FB_U_IRRADIATION      (1ull << 43)

/* 1-D geometry of FillPolar1DArrays (src/SourceEuler.c:71-188) for one
 * process holding all rings (IMIN = 0, GLOBALNRAD = NRAD). */
typedef struct fb_geom {
  int nr, ns;
  double *radii;       /* nr+1 */
  double *rinf;        /* nr+1: Rinf[NRAD] = Radii[NRAD] (SourceEuler.c:118) */
  double *rsup, *rmed, *surf, *invrmed, *invsurf, *invdiffrsup, *invrinf;
  double *invdiffrmed; /* nr, entry 0 stays 0 like the reference's global */
  double *azimuth, *cosaz, *sinaz;  /* ns */
} fb_geom;

int  fb_geom_fill(const fb_params *p, const double *radii, fb_geom *g);
void fb_geom_free(fb_geom *g);

/* Reference helper functions restated on the host with the same
 * expressions (glibc libm is called for the transcendental parts). */
double fb_host_aspect_ratio(const fb_params *p, double r);   /* Viscosity.c:107 */
double fb_host_sigma(const fb_params *p, double r);          /* Theo.c:13      */
double fb_host_energy(const fb_params *p, double r);         /* Theo.c:156     */
double fb_host_smoothing(const fb_params *p, double r);      /* Force.c:255    */

/* POSIX drand48 stream (restated: X <- (0x5DEECE66D X + 0xB) mod 2^48). */
typedef struct { unsigned long long x; } fb_rand48;
void   fb_srand48(fb_rand48 *s, long seed);
double fb_drand48(fb_rand48 *s);

/* GPU helper used by fb_init_state for self-gravity: computes the
 * radial SG acceleration of dens (host array) on the device and returns its
 * azimuthal means (GLOBAL_AxiSGAccr, nr doubles). */
int fb_sg_axisym_accel(fb_ctx *ctx, const double *dens, double *axi_out);
/* Same, for the density already on the device (the context's state). */
int fb_sg_axisym_accel_device(fb_ctx *ctx, double *axi_out);
/* Units of ComputeCodeUnits (src/LowTasks.c:202-229). */
double fb_unit_length(const fb_params *p);
double fb_unit_time(const fb_params *p);         /* LowTasks.c:212 */
double fb_unit_temperature(const fb_params *p);  /* LowTasks.c:213 */
double fb_unit_mass(const fb_params *p);
/* Geometry held by a context (NULL if none). */
const fb_geom *fb_ctx_geom(const fb_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
