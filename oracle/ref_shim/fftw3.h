/* Project-written, CPU-only stand-in for the subset of the FFTW 3 C API that
 * the reference channel-dns sources call (plans: many_dft, many_dft_r2c,
 * many_dft_c2r, many_r2r with REDFT00; new-array execute; threads callback;
 * wisdom and alignment queries).  It restates FFTW's documented transform
 * definitions (unnormalised; forward sign -1, backward +1; REDFT00 as
 * Y_k = x_0 + (-1)^k x_{n-1} + 2 sum_{j=1}^{n-2} x_j cos(pi j k/(n-1))) with a
 * mixed-radix Stockham FFT.  No FFTW code is used.  Test infrastructure only:
 * it exists so the reference's own sources can be compiled here as a checker
 * and CPU baseline.
 */
#ifndef CDNS_FFTW3_SHIM_H
#define CDNS_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct cdns_fftw_plan_s *fftw_plan;

typedef enum {
    FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
    FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
    FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
} fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_UNALIGNED (1U << 1)

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in,
                             const int *inembed, int istride, int idist, fftw_complex *out,
                             const int *onembed, int ostride, int odist, int sign,
                             unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in,
                                 const int *inembed, int istride, int idist, fftw_complex *out,
                                 const int *onembed, int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in,
                                 const int *inembed, int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_many_r2r(int rank, const int *n, int howmany, double *in,
                             const int *inembed, int istride, int idist, double *out,
                             const int *onembed, int ostride, int odist,
                             const fftw_r2r_kind *kind, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags);
fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned flags);

void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_execute_r2r(const fftw_plan p, double *in, double *out);
void fftw_destroy_plan(fftw_plan p);

int fftw_alignment_of(double *p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);
void fftw_threads_set_callback(
    void (*parallel_loop)(void *(*work)(char *), char *jobdata, size_t elsize, int njobs,
                          void *data),
    void *data);
int fftw_import_wisdom_from_filename(const char *filename);
int fftw_export_wisdom_to_filename(const char *filename);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
