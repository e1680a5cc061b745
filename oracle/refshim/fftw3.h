/* Declaration-only stand-in so the reference headers compile for the test
 * oracle; no FFT is linked (the spectral diagnostics are off the hot path). */
#ifndef ORACLE_REFSHIM_FFTW3_H
#define ORACLE_REFSHIM_FFTW3_H
#include <cstddef>
typedef double fftw_complex[2];
typedef struct oracle_fftw_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#endif
