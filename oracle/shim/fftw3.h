/*
 * Minimal FFTW3 declarations so that reference sources which include
 * <fftw3.h> (but whose FFTW calls are commented out or unused on the SH
 * hot path) compile for the test oracle.  No FFTW routine is provided.
 */
#ifndef DSH_ORACLE_FFTW3_STUB_H
#define DSH_ORACLE_FFTW3_STUB_H
typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#endif
