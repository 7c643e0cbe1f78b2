/*
 * Minimal FFTW3-compatible API, written for this project (test infrastructure
 * only).  FFTW itself is not installed on the build or GPU hosts, and the
 * reference's prebuilt Windows FFTW binary is compiled third-party code that
 * is never read or linked.  This header declares exactly the subset of the
 * FFTW 3 double-precision API the reference calls:
 *
 *   src/sip.cpp:27,33,51            fftw_execute_dft_r2c / fftw_execute_dft_c2r
 *   src/fsmeld.cpp:272-283,672-688  fftw_alloc_complex, fftw_plan_dft_{r2c,c2r}_1d
 *   src/fsmeld.cpp:564-568,1062-1073 fftw_free, fftw_destroy_plan
 *
 * Semantics follow FFTW's published documentation: r2c produces the n/2+1
 * non-redundant outputs of the unnormalised forward DFT (sign -1); c2r is the
 * unnormalised inverse (sign +1) of a Hermitian half-spectrum.
 */
#ifndef FSMELD_ORACLE_FFTW3_SHIM_H
#define FSMELD_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fsmeld_shim_plan_s* fftw_plan;

#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE (0U)

fftw_complex* fftw_alloc_complex(unsigned long n);
double* fftw_alloc_real(unsigned long n);
void fftw_free(void* p);

fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex* in, double* out, unsigned flags);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
