// kernels_fixed.cu -- instantiates the fixed-molecule persistent kernels at one
// precision mode: one thread per sim for N = 1..10 atoms, two threads per sim
// for N = 3..10, each also with streamed host-buffer I/O, and the two-thread
// mixed-batch bucket kernels for N = 3..10. Compiled once per mode
// (-DCE_MODE=0..3) so the instantiations build in parallel.
#include "rk45_sim.cuh"

#ifndef CE_MODE
#error "compile with -DCE_MODE=<0..3>"
#endif

#define CE_CAT2(a, b) a##b
#define CE_CAT(a, b) CE_CAT2(a, b)

namespace ce {

FixedKernelFn CE_CAT(fixed_kernel_m, CE_MODE)(int n) {
  switch (n) {
    case 1: return &rk45_fixed_kernel<1, CE_MODE>;
    case 2: return &rk45_fixed_kernel<2, CE_MODE>;
    case 3: return &rk45_fixed_kernel<3, CE_MODE>;
    case 4: return &rk45_fixed_kernel<4, CE_MODE>;
    case 5: return &rk45_fixed_kernel<5, CE_MODE>;
    case 6: return &rk45_fixed_kernel<6, CE_MODE>;
    case 7: return &rk45_fixed_kernel<7, CE_MODE>;
    case 8: return &rk45_fixed_kernel<8, CE_MODE>;
    case 9: return &rk45_fixed_kernel<9, CE_MODE>;
    case 10: return &rk45_fixed_kernel<10, CE_MODE>;
    default: return nullptr;
  }
}

FixedKernelFn CE_CAT(pair_kernel_m, CE_MODE)(int n) {
  switch (n) {
    case 3: return &rk45_pair_kernel<3, CE_MODE>;
    case 4: return &rk45_pair_kernel<4, CE_MODE>;
    case 5: return &rk45_pair_kernel<5, CE_MODE>;
    case 6: return &rk45_pair_kernel<6, CE_MODE>;
    case 7: return &rk45_pair_kernel<7, CE_MODE>;
    case 8: return &rk45_pair_kernel<8, CE_MODE>;
    case 9: return &rk45_pair_kernel<9, CE_MODE>;
    case 10: return &rk45_pair_kernel<10, CE_MODE>;
    default: return nullptr;
  }
}

FixedKernelFn CE_CAT(io_kernel_m, CE_MODE)(int n, bool pair) {
  if (pair) {
    switch (n) {
      case 3: return &rk45_pair_io_kernel<3, CE_MODE>;
      case 4: return &rk45_pair_io_kernel<4, CE_MODE>;
      case 5: return &rk45_pair_io_kernel<5, CE_MODE>;
      case 6: return &rk45_pair_io_kernel<6, CE_MODE>;
      case 7: return &rk45_pair_io_kernel<7, CE_MODE>;
      case 8: return &rk45_pair_io_kernel<8, CE_MODE>;
      case 9: return &rk45_pair_io_kernel<9, CE_MODE>;
      case 10: return &rk45_pair_io_kernel<10, CE_MODE>;
      default: return nullptr;
    }
  }
  switch (n) {
    case 1: return &rk45_fixed_io_kernel<1, CE_MODE>;
    case 2: return &rk45_fixed_io_kernel<2, CE_MODE>;
    case 3: return &rk45_fixed_io_kernel<3, CE_MODE>;
    case 4: return &rk45_fixed_io_kernel<4, CE_MODE>;
    case 5: return &rk45_fixed_io_kernel<5, CE_MODE>;
    case 6: return &rk45_fixed_io_kernel<6, CE_MODE>;
    case 7: return &rk45_fixed_io_kernel<7, CE_MODE>;
    case 8: return &rk45_fixed_io_kernel<8, CE_MODE>;
    case 9: return &rk45_fixed_io_kernel<9, CE_MODE>;
    case 10: return &rk45_fixed_io_kernel<10, CE_MODE>;
    default: return nullptr;
  }
}

PairBucketFn CE_CAT(pair_bucket_kernel_m, CE_MODE)(int n) {
  switch (n) {
    case 3: return &rk45_pair_bucket_kernel<3, CE_MODE>;
    case 4: return &rk45_pair_bucket_kernel<4, CE_MODE>;
    case 5: return &rk45_pair_bucket_kernel<5, CE_MODE>;
    case 6: return &rk45_pair_bucket_kernel<6, CE_MODE>;
    case 7: return &rk45_pair_bucket_kernel<7, CE_MODE>;
    case 8: return &rk45_pair_bucket_kernel<8, CE_MODE>;
    case 9: return &rk45_pair_bucket_kernel<9, CE_MODE>;
    case 10: return &rk45_pair_bucket_kernel<10, CE_MODE>;
    default: return nullptr;
  }
}

}  // namespace ce
