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
  int pimple;       // transient momentum keeps the alpha_u relaxation (ctrl%pimple)
  // energy equation (ctrl_t phase-10 fields)
  int boussinesq;
  double cp, k_cond, tref, beta, gravity[3];
};

// One case of a batched assembly launch: its arrays, its parameters, the
// first block of its share of each launch range, and its per-run flags.
enum BatchRange { RANGE_N = 0, RANGE_F = 1, RANGE_3N = 2, RANGE_ONE = 3 };

struct alignas(16) BatchCase {
  DeviceCase d;
  AsmParams P;
  int blk0[4];      // first block of this case in the N, F, 3N and one-block ranges
  int transient;    // 1: PISO step, 0: SIMPLE iteration
  int time_scheme;  // ctrl.time_scheme
  int has_outflow;
  int ncorr;        // pressure correctors per iteration (1 for SIMPLE)
};

// Device tables of a batched launch: the cases and, per range, the case of
// every block.
struct AsmBatch {
  const BatchCase* cases;
  const int* blk_case[4];
  int nblk[4];
};

enum BatchOp {
  BOP_FILL_APC = 0,
  BOP_GRADIENTS,
  BOP_RHIECHOW_PISO,  // start of a PISO run: the flux from the initial fields
  BOP_BEGIN_ITER,
  BOP_LIMITER,        // arg: component
  BOP_MOMENTUM,       // arg: component
  BOP_MOM_INTERIOR,   // interior faces of all three components (conv_blend = 0)
  BOP_MOM_FINISH,     // arg: component; boundary faces, sources, relaxation
  BOP_APC,
  BOP_RHIECHOW,
  BOP_OUTFLOW,
  BOP_PPE,            // arg: corrector index
  BOP_CORRECT_CELLS,  // arg: corrector index
  BOP_CORRECT_FLUX,   // arg: corrector index
  BOP_DIAG,
  BOP_DIAG_FINALIZE,
  BOP_COUNT
};

int launch_batch_asm(int op, int arg, const AsmBatch& b, cudaStream_t s);

int geometry_setup(DeviceCase& d, const double* x, const int* fptr, const int* fnodes, double* pcen,
                   const AsmParams& P, cudaStream_t s);
int launch_gradients(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
// energy: psi_T (conv_blend > 0), then the row of the temperature equation per cell
int launch_temperature(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
int launch_limiter(const DeviceCase& d, const AsmParams& P, int comp, cudaStream_t s);
int launch_momentum(const DeviceCase& d, const AsmParams& P, int comp, cudaStream_t s);
// conv_blend = 0: launch_mom_interior once per outer iteration, then before
// each component's solve launch_mom_finish(comp) -- the same A, rhs and ap as
// launch_momentum(comp), bit for bit
int launch_mom_interior(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
int launch_mom_finish(const DeviceCase& d, const AsmParams& P, int comp, cudaStream_t s);
int launch_apc(const DeviceCase& d, double div, cudaStream_t s);
int launch_fill(double* a, long n, double v, cudaStream_t s);
int launch_rhiechow(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
int launch_outflow(const DeviceCase& d, cudaStream_t s);
int launch_ppe(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
int launch_correct(const DeviceCase& d, const AsmParams& P, cudaStream_t s);
int launch_diag(const DeviceCase& d, const AsmParams& P, int transient, cudaStream_t s);
int launch_outer_accum(const DeviceCase& d, cudaStream_t s);
int launch_begin_iter(const DeviceCase& d, int transient, int time_scheme, int inlet_ramp, cudaStream_t s);

}  // namespace mgpu
