/*
 * lynx_b200 — C ABI of the B200-native CheFSI eigensolver hot path.
 *
 * Every entry point replaces one reference LYNX interface (cited per function,
 * paths relative to the LYNX source tree).  The ABI uses plain pointers, sizes
 * and status codes only: no C++ or torch types cross it.
 *
 * Conventions (same as the reference):
 *   - Orbitals are column-major Nd x ncol blocks, column stride `ld` >= Nd
 *     (ld = 0 means ld = Nd), grid index i + j*nx + k*nx*ny (x fastest).
 *   - Complex (k-point) arrays are interleaved (re, im) doubles, like
 *     std::complex<double>.
 *   - Operator entry points take DEVICE pointers and run on the context's
 *     stream (lynx_set_stream).  The *_host entry points take host pointers.
 *   - Every call returns LYNX_OK or an error status; lynx_last_error() gives
 *     the message of the last failing call on the calling thread.  Nothing
 *     calls exit(): a CUDA or solver failure is reported, not fatal.
 *   - A context is not re-entrant: calls on one context must not overlap.
 *     Different contexts are independent (no process-wide coefficient caches).
 */
#ifndef LYNX_B200_H
#define LYNX_B200_H

#if defined(__GNUC__)
#define LYNX_API __attribute__((visibility("default")))
#else
#define LYNX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (the reference throws std::runtime_error or exit()s instead,
 * src/solvers/EigenSolver.cpp:633-635,667-670; src/core/gpu_common.cuh:8-15). */
enum {
    LYNX_OK = 0,
    LYNX_ERR_BAD_ARG = 1,
    LYNX_ERR_CUDA = 2,
    LYNX_ERR_OOM = 3,
    LYNX_ERR_CHOL_FAIL = 4,  /* overlap matrix not positive definite (potrf info > 0) */
    LYNX_ERR_EIG_FAIL = 5,   /* subspace eigensolver did not converge (syev info > 0) */
    LYNX_ERR_NONFINITE = 6,  /* NaN/Inf in the eigenvalues or the subspace matrices */
    LYNX_ERR_TIMEOUT = 7,    /* a bounded device-side wait gave up */
    LYNX_ERR_NOT_SETUP = 8,
    LYNX_ERR_UNSUPPORTED = 9,
    LYNX_ERR_BRACKET = 10    /* Fermi level cannot be bracketed */
};

/* Arithmetic of the CheFSI pass. */
enum {
    LYNX_PREC_FP64 = 0,  /* plain FP64 everywhere */
    LYNX_PREC_MIXED = 1  /* FP32 filter + exact int8-slice tensor-core Rayleigh-Ritz products, FP64 subspace algebra */
};

enum { LYNX_BC_PERIODIC = 0, LYNX_BC_DIRICHLET = 1 };
enum { LYNX_SMEAR_GAUSSIAN = 0, LYNX_SMEAR_FERMI_DIRAC = 1 };

typedef struct lynx_ctx lynx_ctx;

LYNX_API const char* lynx_status_string(int status);
LYNX_API const char* lynx_last_error(void);
LYNX_API int lynx_version(void);

/* Grid, lattice and FD stencil of one cell on one device.
 * Replaces FDGrid(Nx,Ny,Nz,lattice,bc...) (src/core/FDGrid.hpp:11-12),
 * Lattice(latvec, cell_type) (src/core/Lattice.hpp:10),
 * FDStencil(order, grid, lattice) (src/operators/FDStencil.hpp:12),
 * HaloExchange(domain, FDn) (src/parallel/HaloExchange.hpp:21) and
 * Hamiltonian::setup / setup_gpu (src/operators/Hamiltonian.hpp:50-54,119-123).
 *   latvec: 3x3 row-major, rows are the lattice vectors (Bohr).
 *   orthogonal: 1 for CellType::Orthogonal, 0 for NonOrthogonal.
 *   bc: 3 ints, LYNX_BC_PERIODIC or LYNX_BC_DIRICHLET per direction (NULL = periodic). */
LYNX_API int lynx_create(lynx_ctx** out, int device, int nx, int ny, int nz, int fd_order, const double* latvec,
                int orthogonal, const int* bc);
LYNX_API int lynx_destroy(lynx_ctx* ctx);

/* CUDA stream (cudaStream_t) for all later work on this context; NULL = the legacy default stream. */
LYNX_API int lynx_set_stream(lynx_ctx* ctx, void* stream);

/* Nd, dV (FDGrid::dV, src/core/FDGrid.cpp:33) and the largest eigenvalue of -0.5*Lap
 * (FDStencil::max_eigval_half_lap, src/operators/FDStencil.cpp:154-180). */
LYNX_API int lynx_grid_info(const lynx_ctx* ctx, int* nd, double* dV, double* max_eigval_half_lap);

/* Scaled stencil coefficients, FDn+1 doubles each (any pointer may be NULL):
 * FDStencil::D2_coeff_{x,y,z}, D2_coeff_{xy,xz,yz}, D1_coeff_{x,y,z} (src/operators/FDStencil.hpp:19-31). */
LYNX_API int lynx_stencil_coeffs(const lynx_ctx* ctx, double* d2x, double* d2y, double* d2z, double* d2xy,
                        double* d2xz, double* d2yz, double* d1x, double* d1y, double* d1z);

/* Nonlocal projector tables, in the flattened form the reference uploads in
 * Hamiltonian::setup_gpu (src/operators/Hamiltonian.cu:342-495) from
 * NonlocalProjector::setup (src/operators/NonlocalProjector.cpp:13-119) and
 * Crystal::compute_nloc_influence (src/atoms/Crystal.cpp:136-255):
 *   n_img images of atoms whose rc-sphere meets the cell; image i belongs to
 *   physical atom img_atom[i], covers img_ndc[i] grid points listed in gpos
 *   (concatenated over images), has lattice shift img_shift[3i..3i+2] (Bohr,
 *   AtomNlocInfluence::image_shift) and projector values chi (concatenated over
 *   images, each block img_ndc[i] x atom_nproj[img_atom[i]] column-major).
 *   gamma: KB energies per (atom, projector) in atom order.
 * Host pointers; the tables are copied to the device. n_img = 0 clears them. */
LYNX_API int lynx_set_nonlocal(lynx_ctx* ctx, int n_img, const int* img_atom, const int* img_ndc,
                      const double* img_shift, const int* gpos, const double* chi, int n_atom,
                      const int* atom_nproj, const double* gamma);

/* Bloch vector for the *_kpt entry points, in the reference's k-point units
 * (KPoints::kpts_cart, src/core/KPoints.cpp:49-52; ghost phase e^{+-i k_d L_d},
 * src/parallel/HaloExchange.cpp:121-133; projector phase e^{-i k.R_image},
 * src/operators/NonlocalProjector.cpp:253-257).
 * Replaces Hamiltonian::set_kpoint_gpu (src/operators/Hamiltonian.hpp:129) and
 * NonlocalProjector::set_kpoint (src/operators/NonlocalProjector.hpp:57). */
LYNX_API int lynx_set_kpoint(lynx_ctx* ctx, const double* kpt_cart);

/* y = H psi + c psi, H = -0.5 Lap + Veff + Vnl.  Device pointers; veff is Nd doubles.
 * Replaces Hamiltonian::apply (src/operators/Hamiltonian.hpp:64-65) / apply_gpu (:137). */
LYNX_API int lynx_hamiltonian_apply(lynx_ctx* ctx, const double* psi, const double* veff, double* y, int ncol, int ld,
                           double c);

/* Complex k-point version. Replaces Hamiltonian::apply_kpt (src/operators/Hamiltonian.hpp:78-80). */
LYNX_API int lynx_hamiltonian_apply_kpt(lynx_ctx* ctx, const double* psi_z, const double* veff, double* y_z, int ncol,
                               int ld, double c);

/* hpsi += Vnl psi.  Replaces NonlocalProjector::apply / apply_kpt
 * (src/operators/NonlocalProjector.hpp:47,51). */
LYNX_API int lynx_nonlocal_apply(lynx_ctx* ctx, const double* psi, double* hpsi, int ncol, int ld);
LYNX_API int lynx_nonlocal_apply_kpt(lynx_ctx* ctx, const double* psi_z, double* hpsi_z, int ncol, int ld);

/* Chebyshev filter of degree `degree`: Y = p_m(H) X with the reference's scaled three-term
 * recurrence.  Replaces EigenSolver::chebyshev_filter_impl (src/solvers/EigenSolver.cpp:559-619)
 * and chebyshev_filter_gpu (src/solvers/EigenSolver.cu:755-783).  `precision` selects FP64 or
 * the FP32 filter; input and output stay FP64. */
LYNX_API int lynx_chebyshev_filter(lynx_ctx* ctx, const double* X, double* Y, const double* veff, int ncol, int ld,
                          double lambda_cutoff, double eigmin, double eigmax, int degree, int precision);
LYNX_API int lynx_chebyshev_filter_kpt(lynx_ctx* ctx, const double* X_z, double* Y_z, const double* veff, int ncol,
                              int ld, double lambda_cutoff, double eigmin, double eigmax, int degree,
                              int precision);

/* One CheFSI pass on device-resident orbitals: filter -> Cholesky-QR -> project -> subspace
 * eigensolve -> rotate.  psi (device, in/out) is overwritten by the Ritz vectors; eig (HOST,
 * nband doubles) receives the Ritz values in ascending order; *lambda_cutoff_out (may be NULL)
 * receives eig[nband-1] + 0.1 (the reference's next cutoff, src/solvers/EigenSolver.cpp:817).
 * Replaces EigenSolver::solve_resident (src/solvers/EigenSolver.hpp:101-104) and, with host
 * data, EigenSolver::solve (:38-41). */
LYNX_API int lynx_eigensolver_solve(lynx_ctx* ctx, double* psi, double* eig, const double* veff, int nband, int ld,
                           double lambda_cutoff, double eigmin, double eigmax, int degree, int precision,
                           double* lambda_cutoff_out);

/* Complex k-point CheFSI pass at the context's k-point (lynx_set_kpoint).
 * Replaces EigenSolver::solve_kpt / solve_kpt_resident (src/solvers/EigenSolver.hpp:49-53,107-110). */
LYNX_API int lynx_eigensolver_solve_kpt(lynx_ctx* ctx, double* psi_z, double* eig, const double* veff, int nband,
                               int ld, double lambda_cutoff, double eigmin, double eigmax, int degree,
                               int precision, double* lambda_cutoff_out);

/* Host-pointer CheFSI pass: EigenSolver::solve (src/solvers/EigenSolver.hpp:38-41) exactly as the
 * CPU caller uses it (psi, eig, Veff in host memory).  Copies in, solves on the device, copies out. */
LYNX_API int lynx_eigensolver_solve_host(lynx_ctx* ctx, double* psi, double* eig, const double* veff, int nband,
                                int ld, double lambda_cutoff, double eigmin, double eigmax, int degree,
                                int precision, double* lambda_cutoff_out);

/* Batched CheFSI passes: nb independent problems (the k-points and spins of one cell, or the
 * cells of an ensemble, on grids of any sizes), problem i on context ctxs[i] with device
 * orbitals psi[i] (complex interleaved when is_kpt[i], at that context's k-point), host
 * eigenvalues eig[i] and device potential veff[i]; the other arrays give each problem's nband,
 * ld, lambda_cutoff, eigmin, eigmax, and lambda_cutoff_out (may be NULL).  The passes run
 * concurrently, one host thread per problem, so give every context its own stream
 * (lynx_set_stream); problems sharing a context or a stream are serialised.  Returns the first
 * failing status (in problem order).  Replaces the reference's loop over (spin, k-point) in
 * SCF::solve_eigenproblem (src/scf/SCF.cpp:383-410) around EigenSolver::solve / solve_kpt. */
LYNX_API int lynx_eigensolver_solve_batch(lynx_ctx** ctxs, int nb, double** psi, double** eig, const double** veff,
                                          const int* nband, const int* ld, const double* lambda_cutoff,
                                          const double* eigmin, const double* eigmax, const int* is_kpt, int degree,
                                          int precision, double* lambda_cutoff_out);

/* Extreme eigenvalue estimates of H by Lanczos (tolerance on both ends, at most max_iter steps,
 * fixed seed), returned with the reference's safety margins (max*1.01, min-0.1).  Device veff.
 * Replaces EigenSolver::lanczos_bounds / lanczos_bounds_kpt (src/solvers/EigenSolver.hpp:43-45,55-58;
 * src/solvers/Lanczos.hpp:92-200). */
LYNX_API int lynx_lanczos_bounds(lynx_ctx* ctx, const double* veff, double tol, int max_iter, double* eigmin,
                        double* eigmax);
LYNX_API int lynx_lanczos_bounds_kpt(lynx_ctx* ctx, const double* veff, double tol, int max_iter, double* eigmin,
                            double* eigmax);

/* Nonlocal forces and energy of device orbitals psi (nband columns, column stride ld; real):
 *   force[3a + d] = -2 occfac sum_n occ[n] sum_p Gamma_p alpha_{p,n} beta_{p,n,d},
 *   *energy_nl    =    occfac sum_n occ[n] sum_p Gamma_p alpha_{p,n}^2,
 * alpha = dV chi^T psi summed over the atom's images, beta_d the same projection of the FD first
 * derivative of psi along lattice direction d.  occ: host, nband occupations; force: host,
 * 3 * n_atom doubles; energy_nl may be NULL.  Replaces Hamiltonian::compute_nonlocal_force_gpu
 * (src/operators/Hamiltonian.hpp:150-153; the formula of src/physics/Forces.cpp:509-797). */
LYNX_API int lynx_nonlocal_force(lynx_ctx* ctx, const double* psi, int nband, int ld, const double* occ, double occfac,
                                 double* force, double* energy_nl);
/* Complex k-point version at the context's k-point: force = -spn_fac_wk sum_n occ sum_p Gamma
 * Re(conj(alpha) beta), energy = (spn_fac_wk / 2) sum_n occ sum_p Gamma |alpha|^2, with the Bloch
 * factors of the nonlocal apply.  Replaces Hamiltonian::compute_nonlocal_force_kpt_gpu
 * (src/operators/Hamiltonian.hpp:163-166). */
LYNX_API int lynx_nonlocal_force_kpt(lynx_ctx* ctx, const double* psi_z, int nband, int ld, const double* occ,
                                     double spn_fac_wk, double* force, double* energy_nl);

/* Start orbitals on the device, as the reference's GPU path draws them: a cuRAND default
 * pseudo-random generator (XORWOW) seeded with `seed` fills nband contiguous columns of Nd
 * doubles (2 Nd for complex, real and imaginary interleaved) with uniform values in (0, 1].
 * The reference seeds (spin s, k-point k) with (spin_start + s) * 1000 + (s * Nkpts + k) * 13 + 1.
 * ld must be Nd or 0.  A fresh generator per call: the same values as the reference's first
 * (spin, k-point) block.  Replaces EigenSolver::randomize_psi_gpu (src/solvers/EigenSolver.hpp:160;
 * src/solvers/EigenSolver.cu:1199-1228) for one block. */
LYNX_API int lynx_randomize_orbitals(lynx_ctx* ctx, double* psi, int nband, int ld, unsigned long long seed,
                                     int is_complex);

/* All (spin, k-point) blocks as EigenSolver::randomize_psi_gpu(Nspin_local, spin_start, Nkpts)
 * draws them (src/solvers/EigenSolver.cu:1199-1228): one generator kept across the blocks,
 * re-seeded per block i = s * nkpts + k with (spin_start + s) * 1000 + i * 13 + 1.  Re-seeding
 * does not rewind the generator's position, so later blocks differ from a fresh generator with
 * the same seed; this entry reproduces the reference's draw for every block.  psi[i]: nband
 * contiguous columns of Nd doubles (2 Nd for complex), i < nspin_local * nkpts. */
LYNX_API int lynx_randomize_orbitals_all(lynx_ctx* ctx, double** psi, int nspin_local, int spin_start, int nkpts,
                                         int nband, int is_complex);

/* Kinetic and nonlocal stress of device psi (nband columns, leading dimension ld), before the
 * division by the cell measure, Voigt order xx, xy, xz, yy, yz, zz:
 *   stress_k[ab]  = -occfac dV sum_n occ[n] <D_a psi_n, D_b psi_n>,
 *   stress_nl[ab] = -2 occfac sum_n occ[n] sum_p Gamma_p alpha_{p,n} beta^{ab}_{p,n} - delta_ab E_nl,
 * D_a the Cartesian FD first derivative, alpha = dV chi^T psi, beta^{ab} = dV sum_g chi(g)
 * (r_g - R_img)_b D_a psi(g) with the Cartesian position relative to the image centre, and
 * E_nl = occfac sum_n occ[n] sum_p Gamma_p alpha^2.  img_pos: host, 3 doubles per image (the
 * image centres of lynx_set_nonlocal, in the grid's coordinates: non-Cartesian for
 * non-orthogonal cells); may be NULL without projectors.  stress_k, stress_nl: host, 6 doubles
 * each.  Replaces Hamiltonian::compute_kinetic_nonlocal_stress_gpu
 * (src/operators/Hamiltonian.hpp:156-160; the formula of src/physics/Stress.cpp:1041-1784). */
LYNX_API int lynx_kinetic_nonlocal_stress(lynx_ctx* ctx, const double* psi, int nband, int ld, const double* occ,
                                          double occfac, const double* img_pos, double* stress_k, double* stress_nl);
/* Complex k-point version at the context's k-point (Bloch factors as in the nonlocal apply),
 * with occfac replaced by spn_fac_wk / 2.  Replaces
 * Hamiltonian::compute_kinetic_nonlocal_stress_kpt_gpu (src/physics/Stress.cpp:967-976). */
LYNX_API int lynx_kinetic_nonlocal_stress_kpt(lynx_ctx* ctx, const double* psi_z, int nband, int ld,
                                              const double* occ, double spn_fac_wk, const double* img_pos,
                                              double* stress_k, double* stress_nl);

/* Fermi level by Brent's method on sum_i w_i f(eps_i - Ef) = nelectron (tolerance 1e-14, <= 200
 * iterations), f Fermi-Dirac or Gaussian smearing.  Host arrays, FP64.
 * Replaces Occupation::find_fermi_level (src/electronic/Occupation.cpp:48-84). */
LYNX_API int lynx_fermi_level(const double* eigs, const double* weights, int n, double nelectron, double beta,
                     int smearing, double* ef);

/* occ[i] = f(eigs[i] - ef).  Replaces the occupation loop of Occupation::compute
 * (src/electronic/Occupation.cpp:208-218) and Occupation::smearing_function (:26-35). */
LYNX_API int lynx_occupations(const double* eigs, int n, double ef, double beta, int smearing, double* occ);

/* Diagnostic, no counterpart in the reference: device time of one Chebyshev degree step
 * (out = a*H*x + b*x + d*xold over ncol columns of this context's grid), averaged over `reps`
 * back-to-back steps on the context's work buffers and timed with CUDA events on the context's
 * stream.  with_nonlocal: 0 = the local step alone; 1 = the whole step with the nonlocal term
 * (projections, expansion and stencil); 2 = the same step, but the time returned is that of
 * the stencil kernel launch alone (the nonlocal term fused into it where it applies), each
 * launch bracketed by its own events. */
LYNX_API int lynx_time_filter_step(lynx_ctx* ctx, const double* veff, int ncol, int precision, int with_nonlocal,
                                   int reps, double* ms_per_step);

/* Rayleigh-Ritz products of the mixed-precision pass on FP32 blocks (device pointers, rows x n,
 * column stride ld; ld and rows multiples of 4, Y and HY 16-byte aligned), on the tensor cores
 * with exact int8 slices and an FP64 result:
 *   Ms = scale * Y^T Y  (N x N column-major; only the upper triangle is guaranteed),
 *   Hs = scale * Y^T HY (N x N column-major, full).
 * Replaces the overlap and projection products of EigenSolver::orthogonalize_gpu /
 * project_and_diag_gpu (src/solvers/EigenSolver.cu:195-233; scale = dV there). */
LYNX_API int lynx_gram_mixed(lynx_ctx* ctx, const float* Y, const float* HY, long long ld, long long rows, int n,
                             double scale, double* Ms, double* Hs);

/* Subspace rotation of the mixed-precision pass: psi = Y W (device pointers; Y FP32 rows x n,
 * column stride ld; W FP64 n x n column-major; psi FP64 rows x n, column stride ldp), on the
 * tensor cores with exact int8 slices.  Ms is the overlap of Y (Ms_ii = scale |y_i|^2, any
 * positive scale): its diagonal sets the per-state power-of-two scaling.  n <= 1551.
 * Replaces EigenSolver::rotate_orbitals_gpu (src/solvers/EigenSolver.cu:312-329). */
LYNX_API int lynx_rotate_mixed(lynx_ctx* ctx, const float* Y, long long ld, long long rows, const double* Ms,
                               const double* W, int n, double* psi, long long ldp);

/* Electron density of one (spin, k-point) block of device orbitals psi (nband columns, stride ld;
 * complex interleaved when is_complex): rho[i] = (accumulate ? rho[i] : 0)
 * + sum_n weight * occ[n] * |psi_n(i)|^2, states with occ[n] < 1e-16 skipped; occ: host, nband
 * doubles; rho: device, Nd doubles; weight = spin factor (2 for one spin channel) x k-point weight.
 * Replaces ElectronDensity::compute for one (spin, k-point) (src/electronic/ElectronDensity.cpp:85-121);
 * the sum over spins and k-points is accumulate = 1 on later blocks. */
LYNX_API int lynx_electron_density(lynx_ctx* ctx, const double* psi, int nband, int ld, const double* occ,
                                   double weight, double* rho, int is_complex, int accumulate);

/* One CheFSI pass of real orbitals, as lynx_eigensolver_solve, for a system of one spin channel and
 * one k-point, followed by the next steps of the SCF iteration on its Ritz values: the Fermi level
 * (Brent on sum_n weight f(eig_n - Ef) = nelectron, smearing as lynx_fermi_level), the
 * occupations, and the electron density rho (device, Nd doubles) = sum_n weight f_n |psi_n|^2 of
 * the new orbitals.  In the mixed-precision pass the tensor-core rotation accumulates the density
 * from the FP64 orbitals as it writes them, so they are not read again.  *ef_out (may be NULL)
 * receives Ef.  Replaces, for one (spin, k-point), EigenSolver::solve -> Occupation::compute ->
 * ElectronDensity::compute in SCF::run (src/physics/SCF.cpp:251-252,433-435). */
LYNX_API int lynx_eigensolver_solve_density(lynx_ctx* ctx, double* psi, double* eig, const double* veff, int nband,
                                            int ld, double lambda_cutoff, double eigmin, double eigmax, int degree,
                                            int precision, double* lambda_cutoff_out, double nelectron, double beta,
                                            int smearing, double weight, double* rho, double* ef_out);

/* ---- Effective potential (the V_eff build of an SCF iteration), FP64, device pointers to fields
 * of Nd points (x fastest), spin-unpolarised. ---- */

/* GGA-PBE exchange-correlation: exc (energy per particle), vxc = d(rho eps)/d rho - div(2
 * d(rho eps)/d sigma lapc_T grad rho), and, when dxcdgrho is not NULL, 2 d(rho eps)/d sigma.  The
 * functional sees rho, or max(rho + rho_core, 1e-14) when rho_core is not NULL; points with a
 * density <= 1e-14 contribute nothing.  Gradients are the FD first derivatives of the context's
 * order with its boundary conditions.  Replaces XCFunctional::evaluate for XCType::GGA_PBE
 * (src/xc/XCFunctional.hpp:41; src/xc/XCFunctional.cpp:193-273), which calls libxc's
 * XC_GGA_X_PBE + XC_GGA_C_PBE; this library evaluates its own restatement of the published
 * functional (PBE 1996 with PW92 correlation). */
LYNX_API int lynx_xc_gga_pbe(lynx_ctx* ctx, const double* rho, const double* rho_core, double* vxc, double* exc,
                             double* dxcdgrho);

/* Poisson equation -Lap phi = rhs by AAR (m = 7 history columns, Anderson every 6th step,
 * omega = beta = 0.6, Jacobi preconditioner), phi the start on entry and the solution on return;
 * stops when ||rhs + Lap phi|| <= tol ||rhs|| (checked after Anderson steps) or after max_iter
 * steps (<= 0: 3000).  *iters (may be NULL) receives the step count.  rhs is used as given: for a
 * periodic cell it must have zero mean.  Replaces PoissonSolver::solve
 * (src/solvers/PoissonSolver.hpp:58; src/solvers/PoissonSolver.cpp:43-159). */
LYNX_API int lynx_poisson_solve(lynx_ctx* ctx, const double* rhs, double* phi, double tol, int max_iter, int* iters);

/* V_eff = V_xc + phi: GGA-PBE as lynx_xc_gga_pbe (rho_core may be NULL), then phi from
 * -Lap phi = 4 pi rho + 4 pi rho_b (rho_b, the pseudocharge, may be NULL) with the right-hand
 * side's mean removed, phi (start on entry) shifted to zero mean.  For a periodic cell the
 * equation is solved by FFT (*poisson_iters = 0) unless LYNX_OPT_POISSON_DIRECT is 0; otherwise,
 * and for Dirichlet directions, by AAR as lynx_poisson_solve.  veff, vxc, exc, phi: Nd
 * doubles each; *poisson_iters may be NULL.  Replaces EffectivePotential::compute for one spin
 * channel without NLCC spinors or mGGA (src/physics/EffectivePotential.hpp:58-66;
 * src/physics/EffectivePotential.cpp:44-177). */
LYNX_API int lynx_effective_potential(lynx_ctx* ctx, const double* rho, const double* rho_b, const double* rho_core,
                                      double poisson_tol, double* veff, double* vxc, double* exc, double* phi,
                                      int* poisson_iters);

/* Diagnostic, no counterpart in the reference: one CTA waits, with at most `spins` tries
 * (1 .. 2^20), for an mbarrier phase that nothing completes, with the same bounded wait the
 * pipelined kernels use for their copies.  The wait gives up and the kernel returns; the call
 * returns LYNX_ERR_TIMEOUT and the context stays usable.  Exercises the timeout error path
 * without a hang. */
LYNX_API int lynx_selftest_wait_timeout(lynx_ctx* ctx, int spins);

/* hpsi += Vnl psi, as lynx_nonlocal_apply, but with no device allocation: the projector
 * coefficients live in a fixed 8 MiB device array inside the library (total projectors x ncol
 * rounded up to 32, in doubles, must fit, else LYNX_ERR_BAD_ARG).  No counterpart in the
 * reference: its GPU path sizes d_alpha once for Nband columns in Hamiltonian::setup_gpu
 * (src/operators/Hamiltonian.cu:473) and has no per-call variant.  The array is shared by all
 * contexts on a device, so calls overlapping in time race; the first call on a device does
 * one-time set-up and should come before any stream capture.  The array's device address is
 * resolved once per device and kept: it does not survive cudaDeviceReset.  Real (Gamma-point)
 * FP64 only. */
LYNX_API int lynx_nonlocal_apply_noalloc(lynx_ctx* ctx, const double* psi, double* hpsi, int ncol, int ld);

/* Execution options of a context (no counterpart in the reference).  The first two compute the
 * same results with either setting, bitwise:
 *   LYNX_OPT_AUTOTUNE:       1 (default) times the compiled stencil launch shapes on the first
 *                            launch for each grid and column count and keeps the fastest; 0 uses
 *                            the default shape.
 *   LYNX_OPT_FUSE_NONLOCAL:  1 (default) adds the nonlocal term inside the stencil kernel when
 *                            the projector spheres are disjoint (real data, periodic orthogonal
 *                            cell, FD order 12), from a compact per-point expansion; 0 always
 *                            uses the separate gather and scatter kernels.
 *   LYNX_OPT_TC_RAYLEIGH_RITZ: 1 (default) runs the mixed-precision pass's Gram products and
 *                            rotation on the tensor cores (exact int8 slices, as accurate as
 *                            FP64 products of the FP32 blocks to about 1e-8); 0 runs them as FP64
 *                            library products on FP64 copies of the FP32 blocks (slower).
 *   LYNX_OPT_COMPACT_GATHER: with the fused nonlocal term, 1 makes every filter step also write
 *                            its output at the sphere points as a compact block, and the next
 *                            step's projections read that block instead of the full grid; 0
 *                            (default) reads the full grid.  Same results, bitwise.
 *   LYNX_OPT_POISSON_DIRECT: 1 (default) makes lynx_effective_potential solve the Poisson equation
 *                            of a periodic cell exactly by FFT (the discrete equation the AAR
 *                            iteration converges to, to rounding); 0 uses the AAR iteration.
 *                            lynx_poisson_solve is always the AAR iteration.
 *   LYNX_OPT_STENCIL_SHAPE:  0 (default) leaves the stencil launch shape to LYNX_OPT_AUTOTUNE;
 *                            k >= 1 makes every pipelined stencil launch use compiled shape k - 1
 *                            (a diagnostic for timing the shapes one by one; an index past the
 *                            compiled shapes selects the default shape, and a shape whose stages
 *                            do not fit the grid fails with LYNX_ERR_UNSUPPORTED).  Same results,
 *                            bitwise.
 *   LYNX_OPT_HOST_COPY_BLOCK: columns per block of the pipelined host-to-device copy of
 *                            lynx_eigensolver_solve_host (mixed precision, >= 256 states): 0 or
 *                            less restores the default (128); the filter starts on a block as
 *                            soon as it has landed.  Same results, bitwise.
 */
enum {
    LYNX_OPT_AUTOTUNE = 1,
    LYNX_OPT_FUSE_NONLOCAL = 2,
    LYNX_OPT_TC_RAYLEIGH_RITZ = 3,
    LYNX_OPT_COMPACT_GATHER = 4,
    LYNX_OPT_POISSON_DIRECT = 5,
    LYNX_OPT_STENCIL_SHAPE = 6,
    LYNX_OPT_HOST_COPY_BLOCK = 7
};
LYNX_API int lynx_set_option(lynx_ctx* ctx, int option, int value);

/* Number of kernel launches this library issued since the last reset (diagnostic counter). */
LYNX_API long long lynx_launch_count(int reset);

#ifdef __cplusplus
}
#endif
#endif /* LYNX_B200_H */
