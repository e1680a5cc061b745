/* Declaration-only stand-in (see fftw3.h in this folder). */
#include "fftw3.h"
