// krylov_poly64.cu -- the mixed form's solvers run in FP64 throughout
// (MGPU_PREC_FP64_POLY): Chebyshev-Jacobi PCG and BiCGStab-Jacobi with FP64
// matrix copy, vectors and SpMV accumulation. Not the parity form (its
// preconditioners are not the reference's); it shows what the FP32 arithmetic
// of the mixed form buys at equal algorithms, and it solves to tolerances the
// FP32 inner solves reach only through refinement. The PCG keeps one Krylov
// stream with x in FP64 and replaces the recursive residual by b - A x only to
// confirm convergence (reliable updates with no intermediate replacement).

#include <algorithm>

#include "krylov_poly.cuh"

namespace mgpu {
extern int g_mixed_occ;  // krylov.cu: the mixed_blocks_per_sm tuning key
namespace {

// OCC: resident blocks per SM the register budget is sized for (the
// mixed_blocks_per_sm tuning key, as for the mixed form's kernels)
template <bool L1, int ELL, int OCC = 2>
__global__ void __launch_bounds__(L1 ? 512 : 256, L1 ? 1 : OCC) k_pcg_poly64(KrylovArgs a, MixedArgsT<double> m) {
  VGrid g = whole_grid(a.bar, a.partials, true);
  pcg_mixed_body<double, L1, ELL, !L1>(a, m, g);
}

template <bool L1, int ELL, int OCC = 2>
__global__ void __launch_bounds__(L1 ? 512 : 256, L1 ? 1 : OCC) k_bicgstab_poly64(KrylovArgs a, MixedArgsT<double> m) {
  VGrid g = whole_grid(a.bar, a.partials, true);
  bicgstab_mixed_body<double, L1, ELL, !L1>(a, m, g);
}

// the grid kernel of an ELL mode at the tuned occupancy (2 to 5 blocks per SM)
#define MGPU_POLY64_PICK(KNAME)                                                   \
  const void* pick_##KNAME(int ell) {                                            \
    switch (std::min(std::max(g_mixed_occ, 2), 5) * 3 + ell) {                   \
      case 5 * 3 + 2: return (const void*)KNAME<false, 2, 5>;                    \
      case 5 * 3 + 1: return (const void*)KNAME<false, 1, 5>;                    \
      case 4 * 3 + 2: return (const void*)KNAME<false, 2, 4>;                    \
      case 4 * 3 + 1: return (const void*)KNAME<false, 1, 4>;                    \
      case 3 * 3 + 2: return (const void*)KNAME<false, 2, 3>;                    \
      case 3 * 3 + 1: return (const void*)KNAME<false, 1, 3>;                    \
      case 2 * 3 + 2: return (const void*)KNAME<false, 2, 2>;                    \
      case 2 * 3 + 1: return (const void*)KNAME<false, 1, 2>;                    \
      default: return (const void*)KNAME<false, 0, 2>;                           \
    }                                                                            \
  }
MGPU_POLY64_PICK(k_pcg_poly64)
MGPU_POLY64_PICK(k_bicgstab_poly64)
#undef MGPU_POLY64_PICK

}  // namespace

int launch_pcg_poly64(const KrylovArgs& a, const MixedArgsT<double>& m, cudaStream_t s) {
  const int ell = ell_mode(m);
  return launch_mixed(ell ? (const void*)k_pcg_poly64<true, 1> : (const void*)k_pcg_poly64<true, 0>,
                      pick_k_pcg_poly64(ell), a, m, s);
}

int launch_bicgstab_poly64(const KrylovArgs& a, const MixedArgsT<double>& m, cudaStream_t s) {
  const int ell = ell_mode(m);
  return launch_mixed(ell ? (const void*)k_bicgstab_poly64<true, 1> : (const void*)k_bicgstab_poly64<true, 0>,
                      pick_k_bicgstab_poly64(ell), a, m, s);
}

}  // namespace mgpu
