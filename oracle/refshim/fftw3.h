/* Stand-in so the reference headers compile for the test oracle.  The three
 * calls the isotropic initialiser makes are implemented by a direct DFT
 * (refshim_fftw.cpp, small test grids only); the spectral diagnostics are not
 * compiled. */
#ifndef ORACLE_REFSHIM_FFTW3_H
#define ORACLE_REFSHIM_FFTW3_H
#include <cstddef>
typedef double fftw_complex[2];
typedef struct oracle_fftw_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#endif
