/*
 * TEST INFRASTRUCTURE (oracle).  Minimal FFTW3 API shim.
 *
 * The reference (PRlgt2020) links FFTW3 (`-lfftw3 -lfftw3_threads`, Makefile:3;
 * version not pinned by the reference) for its Fourier-accelerated gauge
 * fixing (nspt.cc:879,897; plans built at Quenched.cc:827-832).  FFTW3 is not
 * installed in this image, so the oracle build of the reference compiles
 * against this header and links `fftw_shim.c`, a project-written restatement
 * of the published transform FFTW computes:
 *
 *   FFTW_FORWARD :  Y[k] = sum_x X[x] exp(-2 pi i k.x / n)   (unnormalised)
 *   FFTW_BACKWARD:  Y[k] = sum_x X[x] exp(+2 pi i k.x / n)   (unnormalised)
 *
 * over a rank-d row-major array, for the `fftw_plan_many_dft` advanced
 * interface with inembed/onembed == NULL (the only form the reference uses).
 *
 * Only the oracle build of the reference includes this file.  Nothing in the
 * product links it.
 */
#ifndef ORACLE_FFTW_SHIM_H
#define ORACLE_FFTW_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct oracle_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany,
                             fftw_complex *in, const int *inembed,
                             int istride, int idist,
                             fftw_complex *out, const int *onembed,
                             int ostride, int odist,
                             int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);

#ifdef __cplusplus
}
#endif

#endif
