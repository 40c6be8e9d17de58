/* oracle_shim.h -- TEST INFRASTRUCTURE ONLY (the CPU oracle), never product code.
 *
 * Force-included (gcc -include) into every translation unit of the
 * reference sources when they are compiled into the oracle binary under
 * oracle/_ref/.  It does two things and nothing else:
 *
 *  1. Seeds: every `srand48(time(NULL))` of the reference
 *     (Interpret.c:276,375,406, Dsys.c:173) becomes oracle_srand48(), which
 *     reads the seed from the ORACLE_SEED environment variable so that runs
 *     are reproducible.
 *
 *  2. Self-gravity in a single process: the reference's sequential build
 *     links fftw_dummy.c, whose rfftwnd_mpi() does nothing, so self-gravity
 *     is silently zero (fftw_dummy.c:26-28).  With -D_FFTW the sources
 *     include the sequential FFTW 2.1.5 headers (mp.h:20-27) but still call
 *     the MPI entry points rfftw2d_mpi_create_plan / rfftwnd_mpi_local_sizes
 *     / rfftwnd_mpi / rfftwnd_mpi_destroy_plan (split.c:73-82,
 *     sgkernel.c:23-26, sgdens.c:82-85, sgacc.c:39-42, main.c:407-410).
 *     This header declares a one-process stand-in for them; the bodies are
 *     in oracle_fftw_shim.c and call FFTW 2.1.5's own sequential rfftwnd.
 */
#ifndef ORACLE_SHIM_H
#define ORACLE_SHIM_H

void oracle_srand48(long seed);
void oracle_libc_srand48(long seed);
#define srand48(s) oracle_srand48(s)

#ifdef _FFTW
#include <rfftw.h>

typedef struct oracle_rfftwnd_mpi_plan_s *rfftwnd_mpi_plan;

#ifndef FFTW_TRANSPOSED_ORDER
#define FFTW_TRANSPOSED_ORDER 1
#endif
#ifndef FFTW_NORMAL_ORDER
#define FFTW_NORMAL_ORDER 0
#endif

rfftwnd_mpi_plan rfftw2d_mpi_create_plan(int comm, int nx, int ny,
                                         fftw_direction dir, int flags);
void rfftwnd_mpi_local_sizes(rfftwnd_mpi_plan p, int *local_nx,
                             int *local_x_start,
                             int *local_ny_after_transpose,
                             int *local_y_start_after_transpose,
                             int *total_local_size);
void rfftwnd_mpi(rfftwnd_mpi_plan p, int n_fields, fftw_real *local_data,
                 fftw_real *work, int output_order);
void rfftwnd_mpi_destroy_plan(rfftwnd_mpi_plan p);
#endif

#endif
