// fb_sg.cu -- log-polar FFT self-gravity (placeholder until the FFT kernels land).
#include "fb_dev.cuh"

struct fb_sg { int dummy; };

int fb_sg_create(fb_sg **out, const fb_params *p, const fb_geom *g, cudaStream_t s)
{
  (void)p; (void)g; (void)s;
  *out = NULL;
  return FB_ERR_UNSUPPORTED;
}
void fb_sg_destroy(fb_sg *sg) { (void)sg; }
void fb_sg_accel(fb_sg *sg, const KP &k, const double *dens, cudaStream_t s) { (void)sg; (void)k; (void)dens; (void)s; }
void fb_sg_update_velocities(const KP &k, cudaStream_t s) { (void)k; (void)s; }
int fb_sg_launches(const fb_sg *sg) { (void)sg; return 0; }
