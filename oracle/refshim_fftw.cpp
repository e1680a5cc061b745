// refshim_fftw.cpp -- a direct-DFT stand-in for the three FFTW calls of the
// reference's isotropic initialiser (fftw_plan_dft_3d, fftw_execute,
// fftw_destroy_plan), so that generate_full_turbulence (isotropic_ini.cpp)
// runs unmodified in the test oracle.  Test infrastructure only: O(n) work per
// output along each axis, for the small grids of the tests.
//
// Transform: out[x] = sum_t in[t] exp(sign * 2 pi i t.x / n) over the three
// axes of an n0 x n1 x n2 row-major array (n2 fastest), unnormalised, as
// FFTW's fftw_plan_dft_3d defines it.
#include <cmath>
#include <complex>
#include <vector>

#include "refshim/fftw3.h"

struct oracle_fftw_plan_s {
    int n[3];
    fftw_complex *in, *out;
    int sign;
};

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned) {
    return new oracle_fftw_plan_s{{n0, n1, n2}, in, out, sign};
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

void fftw_execute(const fftw_plan p) {
    typedef std::complex<double> cd;
    const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
    const long total = (long)n0 * n1 * n2;
    std::vector<cd> a(total), line, res;
    for (long id = 0; id < total; ++id) a[id] = cd(p->in[id][0], p->in[id][1]);
    const double pi = 3.14159265358979323846;
    for (int axis = 2; axis >= 0; --axis) {
        const int n = p->n[axis];
        const long stride = axis == 2 ? 1 : (axis == 1 ? n2 : (long)n1 * n2);
        std::vector<cd> tw(n);
        for (int m = 0; m < n; ++m) tw[m] = cd(std::cos(2 * pi * m / n), p->sign * std::sin(2 * pi * m / n));
        line.resize(n);
        res.resize(n);
        for (long base = 0; base < total; ++base) {
            // the first element of every line along this axis
            const long c = (base / stride) % n;
            if (c != 0) continue;
            for (int t = 0; t < n; ++t) line[t] = a[base + t * stride];
            for (int x = 0; x < n; ++x) {
                cd s = 0.0;
                for (int t = 0; t < n; ++t) s += line[t] * tw[((long)t * x) % n];
                res[x] = s;
            }
            for (int x = 0; x < n; ++x) a[base + x * stride] = res[x];
        }
    }
    for (long id = 0; id < total; ++id) { p->out[id][0] = a[id].real(); p->out[id][1] = a[id].imag(); }
}
