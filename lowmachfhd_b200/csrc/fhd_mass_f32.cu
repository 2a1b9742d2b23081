// fhd_mass_f32.cu -- the FP32 (mixed-precision) instantiation of the
// multispecies mass-flux kernels of fhd_mass.cu, in a translation unit of
// its own so that it is compiled with FMA contraction: the per-face chi
// iteration, Cholesky factor and noise products are issue-bound multiply-add
// chains, and the FP32 results carry a tolerance, not a bitwise bar.  The
// FP64 kernels stay in fhd_mass.cu, uncontracted, for parity with the FP64
// restatement.
#define FHD_MASS_F32_TU
#include "fhd_mass.cu"
