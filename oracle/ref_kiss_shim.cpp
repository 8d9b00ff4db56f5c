// ref_kiss_shim.cpp -- exposes the reference's own KISS FFT (fftMPI's stripped
// kissfft.h, double precision, src/fftmpi/src/ffttype.h FFT_PRECISION == 2) to the
// tests as a checker of the oracle's DFT.  The header is compiled from where it
// lies in the reference tree by oracle/build_ref.sh; nothing of it is copied here.
#include <stdlib.h>
#include "ffttype.h"
#include "kissfft.h"

extern "C" int ref_kiss_fft(int n, int inverse, const double *in, double *out)
{
    kiss_fft_cfg cfg = kiss_fft_alloc(n, inverse, NULL, NULL);
    if (!cfg) return 1;
    kiss_fft(cfg, (const FFT_DATA *)in, (FFT_DATA *)out);
    free(cfg);
    return 0;
}
