// kernels_atom.cu -- instantiates, at one precision mode (-DCE_MODE=0..3), the
// lane-per-atom kernels: fixed molecule for N = 2..10, the one-launch mixed
// kernel, and the single-bucket kernels for N = 2..10.
#include "rk45_atom.cuh"

#ifndef CE_MODE
#error "compile with -DCE_MODE=<0..3>"
#endif

#define CE_CAT2(a, b) a##b
#define CE_CAT(a, b) CE_CAT2(a, b)

namespace ce {

AtomKernelFn CE_CAT(atom_kernel_m, CE_MODE)(int n) {
  switch (n) {
    case 2: return &rk45_atom_kernel<2, CE_MODE>;
    case 3: return &rk45_atom_kernel<3, CE_MODE>;
    case 4: return &rk45_atom_kernel<4, CE_MODE>;
    case 5: return &rk45_atom_kernel<5, CE_MODE>;
    case 6: return &rk45_atom_kernel<6, CE_MODE>;
    case 7: return &rk45_atom_kernel<7, CE_MODE>;
    case 8: return &rk45_atom_kernel<8, CE_MODE>;
    case 9: return &rk45_atom_kernel<9, CE_MODE>;
    case 10: return &rk45_atom_kernel<10, CE_MODE>;
    default: return nullptr;
  }
}

MixedKernelFn CE_CAT(mixed_kernel_m, CE_MODE)(int n) {
  switch (n) {
    case 0: return &rk45_mixed_kernel<CE_MODE>;
    case 2: return &rk45_bucket_kernel<2, CE_MODE>;
    case 3: return &rk45_bucket_kernel<3, CE_MODE>;
    case 4: return &rk45_bucket_kernel<4, CE_MODE>;
    case 5: return &rk45_bucket_kernel<5, CE_MODE>;
    case 6: return &rk45_bucket_kernel<6, CE_MODE>;
    case 7: return &rk45_bucket_kernel<7, CE_MODE>;
    case 8: return &rk45_bucket_kernel<8, CE_MODE>;
    case 9: return &rk45_bucket_kernel<9, CE_MODE>;
    case 10: return &rk45_bucket_kernel<10, CE_MODE>;
    default: return nullptr;
  }
}

}  // namespace ce
