/*
 * mixgpu.h -- C-ABI of the B200 SIMPLE/PISO pressure-velocity hot path.
 *
 * Plain C types only (no torch, no C++), so a Fortran ISO_C_BINDING interface,
 * ctypes or any other FFI can bind it. Every entry point returns an int status:
 *   0                  success
 *   MGPU_E_ARG   (-1)  invalid argument (null pointer, bad size, bad option)
 *   MGPU_E_CUDA  (-2)  a CUDA runtime call failed (message: mgpu_last_error)
 *   MGPU_E_MESH  (-3)  mesh rejected (bad node/cell reference, zero volume, ...)
 *   MGPU_E_BC    (-4)  boundary specification rejected (same codes as build_bc)
 *   MGPU_E_TIMEOUT(-5) a bounded device wait ran out (kernel returned early)
 *   MGPU_E_NOMEM (-6)  device memory budget exceeded
 * Solver outcomes are reported separately through the reference's own codes
 * (argument `ier` / `ierr`), see each function.
 *
 * Index convention: the mesh and CSR arrays crossing this boundary are 1-based,
 * exactly as the reference's Fortran derived types hold them, so the Fortran
 * side passes its arrays without renumbering. Field arrays are cell-major
 * AoS u(3,ncells) (Fortran column-major), as in fields_t.
 */
#ifndef MIXGPU_H
#define MIXGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGPU_OK 0
#define MGPU_E_ARG (-1)
#define MGPU_E_CUDA (-2)
#define MGPU_E_MESH (-3)
#define MGPU_E_BC (-4)
#define MGPU_E_TIMEOUT (-5)
#define MGPU_E_NOMEM (-6)

/* Boundary type codes: identical values to mod_uns_control.f90:32-56. */
#define MGPU_BC_NONE 0
#define MGPU_BC_WALL 1
#define MGPU_BC_SYMMETRY 2
#define MGPU_BC_VINLET 3
#define MGPU_BC_POUTLET 4
#define MGPU_BC_FARFIELD 5
#define MGPU_BC_SLIPWALL 6
#define MGPU_BC_MASSINLET 7
#define MGPU_BC_OUTFLOW 8
#define MGPU_BC_INTERFACE 9
#define MGPU_BC_VINLET_PARAB 10

#define MGPU_MAXBC 32 /* MAXBC, mod_uns_control.f90:58 */

/* Linear-solver selections. The first value of each is the reference's. */
#define MGPU_PPE_JACOBI 0 /* cg_jacobi  (ppe_precond /= 'ic0')           */
#define MGPU_PPE_IC0 1    /* cg_ic0     (ppe_precond = 'ic0', default)    */
#define MGPU_PPE_ILU0 2   /* PCG with ILU(0) (extension; reference lacks) */
#define MGPU_MOM_ILU0 0   /* bicgstab_ilu0 (the reference's only choice)  */
#define MGPU_MOM_JACOBI 1 /* BiCGStab+Jacobi (extension)                   */

/* Arithmetic form of the Krylov solves. */
#define MGPU_PREC_FP64 0  /* plain FP64, parity form                       */
#define MGPU_PREC_MIXED 1 /* FP32 SpMV/preconditioner inside FP64 refinement */
/* The mixed form's solvers (Chebyshev-Jacobi PCG, BiCGStab-Jacobi) in FP64
 * throughout: not the parity form; isolates what the FP32 arithmetic buys. */
#define MGPU_PREC_FP64_POLY 2

/* One control "bc" line: mirrors bc_spec_t, mod_uns_control.f90:114-145
 * (its thermal plane filters are the MgpuTbcPlane table of MgpuCtrl). */
typedef struct {
  int32_t zone;
  int32_t btype;
  double uvel[3];
  double pval;
  double mdot;
  double umean, uspan, uorigin; /* parabolic inlet profile */
  int32_t uaxis;                /* 1=x 2=y 3=z */
  int32_t has_lid;
  int32_t lid_dir;
  int32_t pad0;
  double lid_coord;
  double lid_vel[3];
  int32_t ttype; /* walls and outlets: 0 adiabatic, 1 fixed T (tval), 2 fixed
                   * heat flux qval into the domain; inlets: T = tval */
  int32_t pad1;
  double tval, qval;
} MgpuBcSpec;

/* One "tbc_plane" control line (parse_tbc_plane, mod_uns_control.f90:1251-
 * 1310): on the wall or outlet zone of bc line `bc` (0-based index into
 * MgpuCtrl.bc), the faces whose centre lies on the plane x[pdir-1] = pcoord
 * (within 1e-4 of the mesh's largest extent) take ttype / tval / qval instead
 * of the zone's; the first matching plane of a zone wins (at most 4 a zone). */
typedef struct {
  int32_t bc;
  int32_t pdir; /* 1=x 2=y 3=z */
  double pcoord;
  int32_t ttype;
  int32_t pad0;
  double tval, qval;
} MgpuTbcPlane;
#define MGPU_MAXTBC 32

/* Control scalars: mirrors ctrl_t, mod_uns_control.f90:148-280. */
typedef struct {
  double rho, mu, alpha_u, alpha_p;
  int32_t outer_max;
  int32_t lin_max;
  double outer_tol, lin_tol;
  double conv_blend, nonorth_corr;
  int32_t ppe_precond; /* MGPU_PPE_* */
  int32_t mom_solver;  /* MGPU_MOM_* */
  int32_t transient, time_scheme;
  double dt;
  int32_t n_time_max, n_correct;
  double body_force[3];
  int32_t inlet_ramp;
  int32_t precision; /* MGPU_PREC_* */
  double mixed_tol;  /* inner FP32 relative tolerance per refinement sweep */
  int32_t nbc;
  int32_t n_outer_iter; /* PIMPLE outer iterations per time step (<= 0: 1) */
  MgpuBcSpec bc[MGPU_MAXBC];
  /* Energy equation (temperature_assembly, mod_uns_simple.f90:1748-2037, the
   * fluid/LTE branch): energy = 1 solves it after the corrections of every
   * outer iteration / time step, with the momentum solver, into the solve
   * slot after the pressure sweeps; 0 skips it (T stays as uploaded, which is
   * the reference's result while T is uniform and no boundary is thermal). */
  int32_t energy;
  int32_t boussinesq; /* 1: -rho*beta*(T - tref)*gravity*V in the momentum rhs */
  double cp, k_cond, tref, beta;
  double gravity[3];
  int32_t ntbc;
  int32_t pad_e;
  MgpuTbcPlane tbc[MGPU_MAXTBC];
} MgpuCtrl;

/* Face-list mesh: mirrors mesh_t/face_t, mod_uns_mesh.f90:17-54. */
typedef struct {
  int32_t nnodes, nfaces, ncells;
  int32_t pad0;
  const double* x;          /* 3*nnodes, x(1:3,node) */
  const int32_t* fnode_ptr; /* nfaces+1, 0-based offsets into fnodes */
  const int32_t* fnodes;    /* node ids, 1-based */
  const int32_t* c0;        /* owner cell, 1-based */
  const int32_t* c1;        /* neighbour cell, 1-based, 0 = boundary */
  const int32_t* zone;      /* face zone id */
} MgpuMesh;

/* Fluent ASCII .cas reader: read_cas (mod_uns_cas_reader.f90:44-523) in the
 * library, for hosts without the Fortran front end. Fills *mesh with arrays
 * owned by *holder (valid until mgpu_cas_free). *ier: 0; 1 file not readable;
 * 6/7 bad node section; 8 bad cell section; 9/10 bad face section; 11 unknown
 * face type; 20 missing sections or faces; 21 node or cell reference out of
 * range. No reference counterpart for the holder: the Fortran reader fills
 * mesh_t itself. */
typedef struct MgpuCasMesh MgpuCasMesh;
int mgpu_cas_read(const char* path, MgpuMesh* mesh, MgpuCasMesh** holder, int* ier);
/* The (45 ...) zone records as "id type\n" lines; *len = full length. */
int mgpu_cas_zone_names(const MgpuCasMesh* holder, char* buf, int cap, int* len);
int mgpu_cas_free(MgpuCasMesh* holder);

/* Per outer iteration (SIMPLE) or time step (PISO) record. Solve slots:
 * 0..2 momentum components, 3.. pressure-correction sweeps, then (energy)
 * the temperature solve; dT_max = max |T - T before the solve|. */
#define MGPU_MAXSOLVE 8
typedef struct {
  int32_t it;
  int32_t itl_max;
  int32_t nsolve;
  int32_t pad0;
  int32_t lin_it[MGPU_MAXSOLVE];
  int32_t lin_ierr[MGPU_MAXSOLVE];
  double lin_res[MGPU_MAXSOLVE];
  double imbal, du_max, dT_max, ressum;
  double umax, cfl_max, t_now;
} MgpuIterRec;

typedef struct MgpuCase MgpuCase;

/* Library version and last error message (thread-local, static storage). */
int mgpu_version(void);
const char* mgpu_last_error(void);
/* Selects the CUDA device used by subsequent mgpu_case_create calls. */
int mgpu_set_device(int device);

/* Case lifetime. Replaces uns_solver_init's work after the .cas/.control have
 * been read (mod_uns_driver.f90:60-239: connectivity :91, geometry :94,
 * build_bc :144, init_fields :147): the mesh is uploaded once and every
 * derived array (connectivity, geometry, CSR pattern, face slot maps,
 * triangular level sets) is built and kept resident in HBM.
 * Returns MGPU_E_BC with *ier set to the build_bc code (10..14) on a bad BC. */
int mgpu_case_create(const MgpuMesh* mesh, const MgpuCtrl* ctrl, MgpuCase** out, int* ier);
int mgpu_case_destroy(MgpuCase* c);
/* Device bytes held by the case (mesh, matrices, fields, work vectors). */
int mgpu_case_device_bytes(const MgpuCase* c, int64_t* bytes);

/* Fields in/out: fields_t (mod_uns_fields.f90:29-79). u is u(3,ncells) AoS,
 * p(ncells), flux(nfaces), gu(3,3,ncells). Any pointer may be NULL to skip
 * that field. The AoS <-> device-plane transposes run on the device (a staging
 * buffer of up to 9*ncells doubles is kept with the case after the first
 * call); each field is one copy to or from the caller's array, and the call
 * returns when every copy is done. Page-locked host arrays copy fastest. */
int mgpu_fields_upload(MgpuCase* c, const double* u, const double* p, const double* flux,
                       const double* u_old, const double* u_old_old);
int mgpu_fields_download(MgpuCase* c, double* u, double* p, double* flux, double* gp,
                         double* gu, double* apc);

/* Steady SIMPLE: simple_run (mod_uns_simple.f90:88-288). Runs at most
 * min(outer_max, nsteps) outer iterations (nsteps <= 0: no cap), stopping early
 * on convergence. log: optional, capacity logcap records; *nrec = records
 * written. *ier: 0, 20 momentum breakdown, 21 PPE breakdown, 60 non-finite. */
int mgpu_simple_run(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier);
/* mgpu_simple_run followed by mgpu_fields_download, for callers that copy the
 * fields back after every call (simple_run_gpu, the coupling loop): the same
 * results, with the copies of gp, gu and apc overlapping the last
 * iteration's pressure solve. Those three are final once that iteration's
 * gradients are formed, and go to the host on a second stream when their
 * arrays are page-locked (pageable arrays, or a run that stops before its
 * last iteration, copy everything at the end). Any output may be NULL. The
 * first call on a case creates that stream and a device buffer of 12 doubles
 * per cell. No reference counterpart: simple_run leaves its fields in
 * memory the host already owns. */
int mgpu_simple_run_fields(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier,
                           double* u, double* p, double* flux, double* gp, double* gu, double* apc);

/* Transient PISO: piso_run_mpi at one rank (mod_uns_simple_mpi.f90:298-571).
 * *ier: 0, 30 transient=false, 31 dt<=0, 33 momentum breakdown, 34 PPE
 * breakdown, 60 non-finite. */
int mgpu_piso_run(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier);

/* Transient PIMPLE: pimple_run_mpi at one rank (mod_uns_simple_mpi.f90:580-850):
 * per time step one history shift, then n_outer_iter outer iterations of the
 * momentum predictor with alpha_u relaxation on top of the time term,
 * apc = ap / alpha_u, gradients and Rhie-Chow fluxes, and n_correct pressure
 * corrections. A record per time step: lin_it/lin_res of the last outer
 * iteration's solves, itl_max and ressum over all of them.
 * *ier: 0, 50 transient=false, 51 dt<=0, 53 momentum breakdown, 54 PPE
 * breakdown, 60 non-finite. */
int mgpu_pimple_run(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier);

/* First non-finite value: nan_scan (mod_uns_simple.f90:2375-2426). field:
 * 1 u_x, 2 u_y, 3 u_z, 4 p, 5 T, 6 T_s; cell 1-based; kind 1 NaN, 2 Inf;
 * *ifin = 0 when every value is finite. */
int mgpu_nan_scan(MgpuCase* c, int* ifin, int* field, int* cell, double* val, int* kind);

/* Stand-alone Krylov solves on a host CSR matrix (1-based row_ptr/col_idx,
 * columns sorted per row, as csr_t in mod_uns_linsolver.f90:27-33). The matrix
 * and vectors are copied to the device, solved there, x copied back.
 * Contract of the reference: (tol, maxit) -> (it, res, ierr) with ierr 0
 * converged, 1 maxit, 2 breakdown, +10 factorisation failure.
 *   method: 0 bicgstab_ilu0 (:148-224), 1 cg_jacobi (:230-291),
 *           2 cg_ic0 (:405-461), 3 BiCGStab+Jacobi, 4 PCG+ILU(0).
 *   norm_mode: 0 = serial solvers (gfortran norm2), 1 = the one-rank
 *           distributed solvers of mod_uns_linsolver_mpi.f90 (sqrt of gdot). */
int mgpu_krylov_solve(int n, const int32_t* row_ptr, const int32_t* col_idx, const double* val,
                      const double* b, double* x, double tol, int maxit, int method,
                      int norm_mode, int* it, double* res, int* ierr);

/* The pressure solver of the mixed-precision and FP64 polynomial forms on a
 * host CSR system (arrays 1-based as in mgpu_krylov_solve; no reference
 * counterpart: it stands in for cg_ic0, mod_uns_linsolver.f90:405-461, with
 * the same contract): PCG with a Chebyshev-Jacobi polynomial of degree
 * cheb_degree (<= 0: the tuning keys, as for a case's pressure solve of n
 * rows; 1: Jacobi).
 *   precision: MGPU_PREC_MIXED (the conjugate-gradient recurrence in FP64:
 *              x, r, p, A p and every dot product; the polynomial applied in
 *              FP32 to an FP32 copy of r with an FP32 copy of A; a true
 *              residual b - A x checked when r converges) or
 *              MGPU_PREC_FP64_POLY (the polynomial in FP64 too).
 *   x: initial guess in, solution out. Converged when |b - A x| / |b| <= tol on
 *   the FP64 residual (ierr 0), else ierr 1 after maxit iterations, 2 on a
 *   breakdown. At most 2^23 rows; every row needs its diagonal entry. */
int mgpu_pcg_poly_solve(int n, const int32_t* row_ptr, const int32_t* col_idx, const double* val,
                        const double* b, double* x, double tol, int maxit, int precision, int cheb_degree,
                        int* it, double* res, int* ierr);

/* Temperature fields (fields_t%T, T_old, T_old_old; cell order), for cases
 * with ctrl.energy: T_old / T_old_old may be NULL (then = T). The download
 * gives T and its Green-Gauss gradient gt(3,ncells) of the last gradient
 * pass (either may be NULL). The reference sets the initial T in its driver
 * (init_T + t_pert sin(pi (x - xmin) / Lx), mod_uns_driver.f90:182-196);
 * here the host uploads it. */
int mgpu_temperature_upload(MgpuCase* c, const double* T, const double* T_old, const double* T_old_old);
int mgpu_temperature_download(MgpuCase* c, double* T, double* gt);

/* y = A x on a host CSR matrix (csr_matvec, mod_uns_linsolver.f90:40-52). */
int mgpu_csr_matvec(int n, const int32_t* row_ptr, const int32_t* col_idx, const double* val,
                    const double* x, double* y);

/* Integer mesh pipeline, bit-exact with the reference:
 * build_connectivity (mod_uns_connectivity.f90:28-108) and build_cell_csr
 * (mod_uns_simple.f90:835-887). Outputs are 1-based like the Fortran arrays.
 * Sizes: cf_ptr ncells+1, cf 2*nint+nbnd, c2c_ptr ncells+1, c2c 2*nint,
 * row_ptr ncells+1, col_idx ncells+2*nint (upper bound; *nnz returned). */
int mgpu_build_connectivity(const MgpuMesh* mesh, int32_t* cf_ptr, int32_t* cf, int32_t* c2c_ptr,
                            int32_t* c2c, int32_t* row_ptr, int32_t* col_idx, int32_t* nnz);

/* Geometry: compute_geometry (mod_uns_geometry.f90:40-92) plus the face
 * weights lf of init_fields (mod_uns_fields.f90:147-157), computed on the
 * device. Sizes: xf,sf 3*nfaces; area,lf nfaces; vol ncells; xc 3*ncells. */
int mgpu_geometry(const MgpuMesh* mesh, double* xf, double* sf, double* area, double* vol,
                  double* xc, double* lf);

/* Reverse Cuthill-McKee cell ordering of the cell graph (no counterpart in the
 * reference, which takes the cell order of the .cas file): new_of_old[c-1] is
 * the new 1-based number of cell c. */
int mgpu_rcm_order(const MgpuMesh* mesh, int32_t* new_of_old);

/* The same reverse Cuthill-McKee order computed on the device (adjacency by
 * radix sort, George-Liu start and Cuthill-McKee levels by level-synchronous
 * BFS, each level sorted by (parent position, degree, index)): equal to
 * mgpu_rcm_order entry for entry. At most 2^24 - 1 cells and 255 neighbours
 * per cell. No counterpart in the reference. */
int mgpu_rcm_order_device(const MgpuMesh* mesh, int32_t* new_of_old);

/* The integer arrays a case builds from its mesh (build_connectivity,
 * mod_uns_connectivity.f90:28-108; build_cell_csr and the pos_of slot maps,
 * mod_uns_simple.f90:835-923; the triangular level sets), 0-based, built on
 * the device (on_device = 1: the path mgpu_case_create takes) or by the host
 * builder (0). sizes[0..3] = cell-face entries, nonzeros, lower and upper
 * levels; every array pointer may be NULL (call once with NULLs for the
 * sizes). Sizes: cf_ptr, row_ptr N+1; cf, cf_slot sizes[0]; col, lt_pos
 * sizes[1]; diag, lo_rows, up_rows N; lo_ptr sizes[2]+1; up_ptr sizes[3]+1. */
int mgpu_mesh_topology(const MgpuMesh* mesh, int on_device, int32_t* sizes, int32_t* cf_ptr, int32_t* cf,
                       int32_t* row_ptr, int32_t* col, int32_t* diag, int32_t* cf_slot, int32_t* lt_pos,
                       int32_t* lo_ptr, int32_t* lo_rows, int32_t* up_ptr, int32_t* up_rows);

/* One stage of the outer iteration on the case's current fields, for
 * element-wise checks of each kernel: what = 0 compute_gradients, 1..3
 * momentum_assembly of component what (A values, rhs, ap out), 4 flux_rhiechow,
 * 5 ppe_assembly (A values, rhs out), 6 correct_fields with p' = pp.
 * ts_order sets fields_t%ts_order; apc (optional) replaces the stored apc.
 * aval has room for the CSR pattern (nnz values, mgpu_build_connectivity order). */
int mgpu_case_stage(MgpuCase* c, int what, int ts_order, const double* apc, double* aval, double* rhs,
                    double* ap, const double* pp);

/* Allocation-free PCG with Jacobi preconditioning, for callers that cannot
 * allocate device memory: a host that owns every device byte and passes only
 * its own buffers, or a CUDA Fortran host whose arrays already live on the
 * GPU. No counterpart in the reference, whose solvers allocate their work
 * arrays on every call. The call waits for its stream (it reads the result
 * back to the host), so it does not belong inside a stream capture.
 * Same algorithm and outputs as mgpu_krylov_solve(method 1), but every array
 * is a device pointer (CSR 0-based: row_ptr[0] = 0) and the work space is one
 * fixed array inside the library (about 4.9 MB per GPU that loads it):
 *   - n above MGPU_NOALLOC_MAX_ROWS is rejected with MGPU_E_ARG;
 *   - calls that overlap on the GPU race on that array: serialise them;
 *   - the first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress) once for that device;
 *   - the solve's grid may hold at most 2048 blocks (reduction partials in
 *     the array); a larger one is refused with MGPU_E_ARG.
 * stream: a cudaStream_t (NULL = default). */
#define MGPU_NOALLOC_MAX_ROWS 131072
int mgpu_cg_jacobi_noalloc(int n, const int32_t* d_row_ptr, const int32_t* d_col_idx, const double* d_val,
                           const double* d_b, double* d_x, double tol, int maxit, int norm_mode, void* stream,
                           int* it, double* res, int* ierr);

/* Launch tunables, process-wide (for autotuning): "single_block_rows" (a
 * solve of at most this many rows runs in one block, default 32768),
 * "sweep_threads" (threads of a sync-free triangular sweep, default 65536),
 * "sweep_sleep_ns" (back-off of a long wait in that sweep, default 0),
 * "min_blocks" (least number of blocks of a multi-block solve, default 1),
 * "cheb_degree" (mixed form: degree of the Chebyshev-Jacobi pressure
 * preconditioner, 1 = plain Jacobi, default 24), "cheb_ratio" (lambda_max over
 * lambda_min of its interval, default 1000), "cheb_large_rows",
 * "cheb_degree_large", "cheb_ratio_large" (pressure systems of at least that
 * many rows take that degree and ratio instead; defaults 1048576, 48, 10000;
 * 0 rows: never), "batch_reserve_blocks" (block
 * slots a batched launch leaves free for other streams, so a case being set
 * up while a batch steps is not held up behind its persistent kernels,
 * default 0), "stream_pool" (create this many streams for cases and batches
 * now: creating one later waits for kernels on other streams),
 * "l2_prefetch_mb" (mixed form: a system, or the systems of a batched phase
 * together, streaming more than this many MB per SpMV pass prefetch each
 * tile's successor into L2, default 96), "mixed_blocks_per_sm" (mixed and FP64
 * polynomial single-system solves: 2-8 resident blocks of 256 threads per SM
 * (the FP64 polynomial form 2-5), the register budget sized to match,
 * default 5), "batch_blocks_per_sm" (the
 * same for batched lanes, default 4; set before building a batch),
 * "spin_limit" (failed polls
 * after which a grid-barrier wait gives up, 0 = the built-in bound of about
 * 2 s; for tests of the timeout path), "gather_faces" (assembly kernels: the
 * faces of a cell whose loads a thread issues before summing, 1, 2, 3 or 6
 * (4 and 5 take 3); 0, the default, gives each kernel its measured best;
 * results are the same bits for every value), "barrier_poll_ns" (sleep between two
 * polls of a grid-barrier wait, 0-10000 ns, default 100; 0 polls back to back
 * and backs off by 64 ns after 256 polls). */
int mgpu_set_tuning(const char* key, int value);
/* The value in effect of a mgpu_set_tuning key (every key but stream_pool),
 * e.g. the Chebyshev degree a byte model of the mixed pressure solve needs. */
int mgpu_get_tuning(const char* key, int* value);

/* Coupled mode (the coupling driver's hook, mod_mix_driver.f90:1032 calling
 * uns_solver_step with interface data). A zone given a bc line of type
 * MGPU_BC_INTERFACE is a coupling surface (the reference groups the faces of
 * its "interface" zones the same way, mod_uns_bc.f90:282-323).
 * mgpu_interface_set: set_interface_vel / set_interface_p
 * (mod_uns_bc.f90:730-760): faces 1-based, u(3,n) and p(n) either may be
 * NULL; the values stay with the case until set again (zero at creation).
 * mgpu_interface_mode: set_iface_p_dirichlet (mod_uns_bc.f90:810-813): 0 the
 * peer supplies the face velocity (pressure zero-gradient), 1 it supplies the
 * face pressure (velocity extrapolated; pressure-Dirichlet in the SIMPLE
 * pressure correction; the transient drivers' ppe_assembly_mpi keeps only
 * pressure outlets and far fields Dirichlet, as in the reference).
 * mgpu_interface_set_T: set_interface_T / set_interface_q /
 * set_interface_T_mode (mod_uns_bc.f90:750-793) for a case with the energy
 * equation: per listed face (1-based) the peer's temperature, its heat flux
 * into the domain and the mode (0: Dirichlet T_face = T, 1: Neumann with that
 * flux; bc_face_T, mod_uns_bc.f90:671-696); T, q and mode each may be NULL;
 * zero at creation (Dirichlet at 0, as bcs%iface_T is allocated).
 * mgpu_interface_extract: uns_solver_extract_iface (mod_uns_driver.f90:274-
 * 330) for fluid owner cells: every interface face (bc order, then face
 * order), 1-based, with its owner cell's u(3), p and T; *n = their number (at
 * most cap written); u, p and T each may be NULL. Density (ctrl.rho) is the
 * caller's. The slip, zhang and LTNE interface variants are not provided. */
int mgpu_interface_set(MgpuCase* c, int n, const int32_t* faces, const double* u, const double* p);
int mgpu_interface_set_T(MgpuCase* c, int n, const int32_t* faces, const double* T, const double* q,
                         const int32_t* mode);
int mgpu_interface_mode(MgpuCase* c, int p_dirichlet);
int mgpu_interface_extract(MgpuCase* c, int cap, int32_t* faces, double* u, double* p, double* T, int* n);

/* Timing of the last run on the case's stream (CUDA events): total device ms
 * and, for the dominant kernel family, launches and summed device ms. */
typedef struct {
  double total_ms;
  int64_t spmv_launches;
  double spmv_ms;
  int64_t krylov_launches;
  double krylov_ms;
  int64_t gpu_launches; /* kernels this library launched during the run */
} MgpuTiming;
int mgpu_case_timing(const MgpuCase* c, MgpuTiming* t);
/* Device time (ms) of each Krylov solve of the last profiled run, in launch
 * order (per outer iteration: momentum x, y, z, then the pressure
 * correction(s)); *n = number of solves recorded (at most cap written). */
int mgpu_case_solve_times(const MgpuCase* c, double* ms, int cap, int* n);
/* 1 = record CUDA events around every Krylov-kernel launch of later runs. */
int mgpu_case_set_profiling(MgpuCase* c, int on);

/* ---- Batched runs (no counterpart in the reference, which advances one case
 * per process through simple_run / piso_run_mpi) ------------------------------
 * A batch advances many resident cases of uneven size together, one outer
 * iteration (SIMPLE) or time step (PISO) per step: each assembly kernel is one
 * launch over all members, each Krylov phase of the mixed-precision members is
 * one persistent launch split into lanes (width 1 block for small systems,
 * several blocks for large ones), and an iteration is replayed from a CUDA
 * graph. A member's iteration records, ier codes and fields are those of the
 * same run made through mgpu_simple_run / mgpu_piso_run, within the tolerance
 * of its precision; with a fixed lane policy the result of a member does not
 * depend on the other members. A case belongs to any number of batches, but
 * only one may step it at a time, and a case must not be run by
 * mgpu_simple_run / mgpu_piso_run while a batch steps it. */
typedef struct MgpuBatch MgpuBatch;

/* Start a run of a case for batched stepping: mode 0 = SIMPLE (at most
 * min(outer_max, nsteps) iterations), 1 = PISO (min(n_time_max, nsteps) time
 * steps; ier 30 / 31 and no run as mgpu_piso_run). nsteps <= 0: the ctrl
 * limit alone. The case then advances only in mgpu_batch_step. */
int mgpu_case_begin(MgpuCase* c, int mode, int nsteps, int* ier);
/* After the run has ended (converged, failed or at its limit): the records
 * and ier exactly as mgpu_simple_run / mgpu_piso_run return them. */
int mgpu_case_finish(MgpuCase* c, MgpuIterRec* log, int logcap, int* nrec, int* ier);

int mgpu_batch_create(MgpuCase* const* cases, int ncases, MgpuBatch** out);
int mgpu_batch_destroy(MgpuBatch* b);
/* Lane policy. The mixed-precision solves give bit-identical results on any
 * number of blocks, so the policy only affects speed: systems of more than
 * split_rows rows (at most 32768) run on wide_lanes wide lanes sharing their
 * class's blocks, smaller ones on single-block lanes; lanes take systems from
 * per-class queues at run time. (0, 0) = autotune: the first step times the
 * first pressure solve under each candidate pair and keeps the fastest
 * (default). */
int mgpu_batch_set_policy(MgpuBatch* b, int split_rows, int wide_lanes);
/* Advance every running member by up to iters iterations / steps; returns
 * after the device is done. *active = members still running. */
int mgpu_batch_step(MgpuBatch* b, int iters, int* active);
/* done[k] = 1 when member k has no run in progress. */
int mgpu_batch_poll(MgpuBatch* b, int* done);
/* begin (mode[k]) + step until every member has ended + finish; nrec and ier
 * per member (ier as mgpu_simple_run / mgpu_piso_run). */
int mgpu_batch_run(MgpuBatch* b, const int* mode, int nsteps, int* nrec, int* ier);
typedef struct {
  int32_t ncases;
  int32_t split_rows, wide_lanes;            /* lane policy in use */
  int32_t autotuned;                         /* 1: policy picked by the autotuner */
  int32_t graph;                             /* 1: iterations replay a CUDA graph */
  int32_t lanes, blocks;                     /* first pressure phase: lanes, blocks of its widest launch */
  int32_t launches_per_iter;                 /* kernels one iteration launches */
  double tune_ms;                            /* device time spent by the autotuner */
  double step_ms;                            /* device time of all steps */
  int64_t iters;                             /* iterations stepped */
  /* profiled steps only (mgpu_batch_set_profiling): summed device ms of the
   * Krylov phases (momentum x, y, z, pressure correctors 1..5), of the
   * assembly launches, and of the busiest and the average lane of the
   * first pressure phase (lane time = its first block's start to end) */
  double phase_ms[8];
  double asm_ms;
  double lane_max_ms, lane_mean_ms;
  int64_t profiled_iters;
  int64_t gpu_launches; /* kernels the batch has run (a CUDA graph replay counts its kernels) */
} MgpuBatchInfo;
/* 1 = later steps run launch by launch (no graph) with CUDA events around
 * every phase and lane timestamps (mgpu_batch_info reports them). */
int mgpu_batch_set_profiling(MgpuBatch* b, int on);
int mgpu_batch_info(const MgpuBatch* b, MgpuBatchInfo* info);
/* The lane plan (host only, no GPU needed) of systems of rows[i] rows and
 * passes[i] SpMV-sized passes (NULL: modelled) under a policy and a
 * co-resident block capacity: sys_class[i] = the class (queue) of system i,
 * classes numbered widest lanes first, the last one the single-block lanes;
 * lane_width[0 .. *nlanes) = the lanes' widths, in class order (room for
 * `capacity` entries). */
int mgpu_batch_plan(int nsys, const int* rows, const double* passes, int split_rows, int wide_lanes, int capacity,
                    int* sys_class, int* lane_width, int* nlanes);

#ifdef __cplusplus
}
#endif
#endif
