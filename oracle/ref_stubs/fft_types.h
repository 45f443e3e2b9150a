// Stand-in for the Charm-FFT library's fft_types.h (not in the reference
// tree); the oracle's PINY files include it but use none of its types.
#ifndef OA_REF_STUB_FFT_TYPES_H
#define OA_REF_STUB_FFT_TYPES_H
#include "ckcomplex.h"
// g-point of the density sphere as cp_hart_ext.C reads it: d3 = kx,
// d2 = ky, d1 = kz, offset = index into the rho(g) / vks(g) arrays.
struct gridPoint {
  int d1, d2, d3;
  int offset;
};
#endif
