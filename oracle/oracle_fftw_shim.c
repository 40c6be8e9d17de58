/* oracle_fftw_shim.c -- TEST INFRASTRUCTURE ONLY (the CPU oracle).
 *
 * One-process stand-in for the four FFTW-MPI entry points the reference
 * calls for its log-polar self-gravity (split.c:73-82, sginit.c:59-64,
 * sgkernel.c:23-26, sgdens.c:82-85, sgacc.c:39-42).  With one process the
 * whole (2*Nr) x Ns transform is local, so each call maps onto FFTW 2.1.5's
 * sequential in-place rfftwnd:
 *   local_nx = 2*Nr, local_x_start = 0, total_local_size = 2*Nr*2*(Ns/2+1).
 * FFTW_TRANSPOSED_ORDER only changes where the complex coefficients sit;
 * the reference multiplies spectra element by element over arrays that
 * share one layout (sgacc.c:25-38) and transforms back with the same flag,
 * so the product and the back-transform are the same in either order.
 * Plans use FFTW_ESTIMATE instead of FFTW_MEASURE so that the oracle does
 * the same arithmetic on every run.
 */
#include <stdio.h>
#include <stdlib.h>
#include <rfftw.h>
#include "oracle_shim.h"

struct oracle_rfftwnd_mpi_plan_s {
  rfftwnd_plan seq;
  int nx, ny;
  fftw_direction dir;
};

/* Seeds libc's drand48 stream directly (used by harness.c, whose own
   srand48 name is taken by the macro in oracle_shim.h). */
void oracle_libc_srand48(long seed)
{
  (srand48)(seed);
}

void oracle_srand48(long seed)
{
  const char *s = getenv("ORACLE_SEED");
  (void)seed;
  /* srand48 here is libc's: the macro in oracle_shim.h is not applied to
     this file's own call below because of the parentheses. */
  (srand48)(s ? atol(s) : 0L);
}

rfftwnd_mpi_plan rfftw2d_mpi_create_plan(int comm, int nx, int ny,
                                         fftw_direction dir, int flags)
{
  struct oracle_rfftwnd_mpi_plan_s *p = malloc(sizeof *p);
  (void)comm; (void)flags;
  if (!p) { fprintf(stderr, "oracle fftw shim: out of memory\n"); exit(1); }
  p->nx = nx;
  p->ny = ny;
  p->dir = dir;
  p->seq = rfftw2d_create_plan(nx, ny, dir, FFTW_ESTIMATE | FFTW_IN_PLACE);
  if (!p->seq) { fprintf(stderr, "oracle fftw shim: plan failed\n"); exit(1); }
  return p;
}

void rfftwnd_mpi_local_sizes(rfftwnd_mpi_plan p, int *local_nx,
                             int *local_x_start,
                             int *local_ny_after_transpose,
                             int *local_y_start_after_transpose,
                             int *total_local_size)
{
  *local_nx = p->nx;
  *local_x_start = 0;
  *local_ny_after_transpose = p->ny / 2 + 1;
  *local_y_start_after_transpose = 0;
  *total_local_size = p->nx * 2 * (p->ny / 2 + 1);
}

void rfftwnd_mpi(rfftwnd_mpi_plan p, int n_fields, fftw_real *local_data,
                 fftw_real *work, int output_order)
{
  (void)n_fields; (void)work; (void)output_order;
  if (p->dir == FFTW_REAL_TO_COMPLEX)
    rfftwnd_one_real_to_complex(p->seq, local_data, NULL);
  else
    rfftwnd_one_complex_to_real(p->seq, (fftw_complex *)local_data, NULL);
}

void rfftwnd_mpi_destroy_plan(rfftwnd_mpi_plan p)
{
  if (!p) return;
  rfftwnd_destroy_plan(p->seq);
  free(p);
}
