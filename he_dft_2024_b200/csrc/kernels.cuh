// kernels.cuh -- every device header of libhedft.so.
//
// The host translation units (he_dft.cu, he_noalloc.cu) include it as it is: they see the heavy
// kernel templates (k_stencil, the FFT passes) as declarations only and define the light
// kernels.  The kernel translation units that build.py writes define HE_KERNEL_TU first: they see
// the heavy kernels' bodies, hide the light ones, and explicitly instantiate exactly the heavy
// kernels that the host objects launch (their undefined kernel symbols), several units compiled
// in parallel.
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include "fft_kernels.cuh"
#include "fft_reg.cuh"
#include "fft_xy.cuh"
#include "fft_yz.cuh"
#include "ops.cuh"
#include "setup.cuh"
#include "quantum.cuh"
#include "alphas.cuh"
