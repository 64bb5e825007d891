// krylov_poly64.cu -- the mixed form's solvers run in FP64 throughout
// (MGPU_PREC_FP64_POLY): Chebyshev-Jacobi PCG and BiCGStab-Jacobi with FP64
// matrix copy, vectors and SpMV accumulation. Not the parity form (its
// preconditioners are not the reference's); it shows what the FP32 arithmetic
// of the mixed form buys at equal algorithms, and it solves to tolerances the
// FP32 inner solves reach only through refinement. The PCG keeps one Krylov
// stream with x in FP64 and replaces the recursive residual by b - A x only to
// confirm convergence (reliable updates with no intermediate replacement).

#include "krylov_poly.cuh"

namespace mgpu {
namespace {

template <bool L1, int ELL>
__global__ void __launch_bounds__(L1 ? 512 : 256, L1 ? 1 : 2) k_pcg_poly64(KrylovArgs a, MixedArgsT<double> m) {
  VGrid g = whole_grid(a.bar, a.partials);
  pcg_mixed_body<double, L1, ELL, !L1>(a, m, g);
}

template <bool L1, int ELL>
__global__ void __launch_bounds__(L1 ? 512 : 256, L1 ? 1 : 2) k_bicgstab_poly64(KrylovArgs a, MixedArgsT<double> m) {
  VGrid g = whole_grid(a.bar, a.partials);
  bicgstab_mixed_body<double, L1, ELL, !L1>(a, m, g);
}

}  // namespace

int launch_pcg_poly64(const KrylovArgs& a, const MixedArgsT<double>& m, cudaStream_t s) {
  switch (ell_mode(m)) {
    case 2:
      return launch_mixed((const void*)k_pcg_poly64<true, 1>, (const void*)k_pcg_poly64<false, 2>, a, m, s);
    case 1:
      return launch_mixed((const void*)k_pcg_poly64<true, 1>, (const void*)k_pcg_poly64<false, 1>, a, m, s);
    default:
      return launch_mixed((const void*)k_pcg_poly64<true, 0>, (const void*)k_pcg_poly64<false, 0>, a, m, s);
  }
}

int launch_bicgstab_poly64(const KrylovArgs& a, const MixedArgsT<double>& m, cudaStream_t s) {
  switch (ell_mode(m)) {
    case 2:
      return launch_mixed((const void*)k_bicgstab_poly64<true, 1>, (const void*)k_bicgstab_poly64<false, 2>, a, m, s);
    case 1:
      return launch_mixed((const void*)k_bicgstab_poly64<true, 1>, (const void*)k_bicgstab_poly64<false, 1>, a, m, s);
    default:
      return launch_mixed((const void*)k_bicgstab_poly64<true, 0>, (const void*)k_bicgstab_poly64<false, 0>, a, m, s);
  }
}

}  // namespace mgpu
