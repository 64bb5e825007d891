// assembly.cuh -- case-constant parameters and launchers of the face-loop kernels.
#pragma once

#include "case.cuh"

namespace mgpu {

struct AsmParams {
  double rho, mu, alpha_u, alpha_p, conv_blend, nonorth_corr, dt;
  double body_force[3];
  double flux_ref;      // rho*uscale*area_btot (simple_run :117-130)
  double min_cbrt_vol;  // min over cells of vol**(1/3) (CFL estimate)
  double outer_tol;
  int has_body_force;
  int has_pdir;     // any pressure-Dirichlet boundary face: no PPE pin
  int has_outflow;  // any outflow zone: global outflow rescale
  int inlet_ramp;
};

int geometry_setup(DeviceCase& d, const double* x, const int* fptr, const int* fnodes, double* pcen,
                   const AsmParams& P, cudaStream_t s);
int launch_gradients(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
int launch_limiter(const DeviceCase& d, const AsmParams& P, int comp, cudaStream_t s);
int launch_momentum(const DeviceCase& d, const AsmParams& P, int comp, cudaStream_t s);
int launch_apc(const DeviceCase& d, double div, cudaStream_t s);
int launch_fill(double* a, long n, double v, cudaStream_t s);
int launch_rhiechow(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
int launch_outflow(const DeviceCase& d, cudaStream_t s);
int launch_ppe(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
int launch_correct(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
int launch_diag(const DeviceCase& d, const AsmParams& P, int transient, cudaStream_t s);
int launch_begin_iter(const DeviceCase& d, int transient, int time_scheme, cudaStream_t s);

}  // namespace mgpu
