/* cpphf_b200.h - C ABI of the B200 (sm_100a) Fock-build library.
 *
 * Drop-in device back end for cpp_hf's native operator module
 * (cpp/cpp_hf_native.cpp of skilledwolf/cpp_hf).  Every entry point takes plain
 * device pointers and sizes, runs on the given CUDA stream (NULL = legacy
 * default stream), never allocates device memory (callers pass workspace
 * sized by the matching *_workspace_bytes query) and returns a status code:
 *
 *   CPPHF_OK (0), CPPHF_ERR_INVALID (-1, maps to ValueError),
 *   CPPHF_ERR_CUDA (-2), CPPHF_ERR_TIMEOUT (-3, a bounded device wait gave up),
 *   CPPHF_ERR_NONFINITE (-4), CPPHF_ERR_UNSUPPORTED (-5).
 *
 * cpphf_last_error() returns the calling thread's last error text.
 *
 * Complex arrays are interleaved complex128 (double re, double im), C order,
 * with the (nk1, nk2, nb, nb) layout of the reference (channel index fastest).
 */
#ifndef CPPHF_B200_H
#define CPPHF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CPPHF_ABI_VERSION 1

#define CPPHF_OK 0
#define CPPHF_ERR_INVALID -1
#define CPPHF_ERR_CUDA -2
#define CPPHF_ERR_TIMEOUT -3
#define CPPHF_ERR_NONFINITE -4
#define CPPHF_ERR_UNSUPPORTED -5

const char* cpphf_last_error(void);
int cpphf_version(void);

/* Device error word.  A bounded in-kernel wait that gives up (an mbarrier wait
 * on an asynchronous copy: bit 1; a grid barrier of a cooperative kernel:
 * bit 2) ORs its code into one word per device and the kernel returns early,
 * leaving its outputs incomplete.  The entry points that synchronise (the
 * solvers, cpphf_density_from_fock) read and clear the word before returning
 * and report a set word as CPPHF_ERR_TIMEOUT.  Asynchronous entry points
 * (cpphf_exchange, cpphf_build_fock, cpphf_find_mu_bisection, ...) return
 * before their kernels run, so a timeout of theirs is seen by the next such
 * read or by cpphf_device_error(), which synchronises the device, returns the
 * word (0 = none) and clears it if clear != 0.  The mu kernels also write NaN
 * to mu_out when their barrier gives up.  No counterpart in the reference,
 * whose loops cannot hang (cpp_hf_native.cpp:58-70 maps its C++ exceptions). */
int cpphf_device_error(int clear);

/* Poll limit of the grid barriers in the cooperative mu kernels (each poll an
 * L2 round trip; the default, 2e7, is seconds).  polls <= 0 restores the
 * default.  Process-wide; read at each launch.  Small limits make a barrier
 * give up before slower blocks arrive, which is how the timeout path is
 * tested without hanging a GPU.  No counterpart in the reference. */
int cpphf_set_barrier_spin_limit(long long polls);
long long cpphf_barrier_spin_limit(void);

/* Synchronous host <-> device copies on `stream` (for projector callbacks). */
int cpphf_copy_d2h(void* dst_host, const void* src_device, size_t bytes, void* stream);
int cpphf_copy_h2d(void* dst_device, const void* src_host, size_t bytes, void* stream);

/* ------------------------------------------------------------------------
 * Exchange self-energy.  Replaces _native.selfenergy_fft_full
 * (cpp/cpp_hf_native.cpp:246-278 -> selfenergy.hpp:83-171).
 *   Sigma = -IFFT2[FFT2(P - refP) * VR], VR of orbital width dv (1 or nb);
 *   hcp = Hermitian upper-triangle packing (requires dv == 1);
 *   apply_ifftshift as selfenergy.hpp:174-190; precision 64 (complex128
 *   throughout) or 32 (complex64 FFT, complex128 in/out).
 *   refP may be NULL; Sigma may alias P.
 * ---------------------------------------------------------------------- */
size_t cpphf_exchange_workspace_bytes(int64_t nk1, int64_t nk2, int64_t nb, int hcp,
                                      int precision);
int cpphf_exchange(const void* P, const void* refP, const void* VR, void* Sigma, int64_t nk1,
                   int64_t nk2, int64_t nb, int64_t dv, int hcp, int apply_ifftshift,
                   int precision, void* workspace, size_t workspace_bytes, void* stream);
/* Replaces _native.clear_fft_plan_cache (cpp_hf_native.cpp:280-284).  Plans
 * hold no device memory here (twiddles are built per block), so it is a no-op. */
int cpphf_clear_fft_plan_cache(void);

/* ------------------------------------------------------------------------
 * Batched Hermitian eigendecomposition.  Replaces _native.eigh_batched
 * (cpp_hf_native.cpp:287-312 -> linalg.hpp:39-66): hermitise, then ascending
 * eigenvalues w (batch, nb) and eigenvector columns V (batch, nb, nb).
 * Cyclic complex Jacobi, one warp (nb <= 16) or one CTA per matrix.
 * ---------------------------------------------------------------------- */
int cpphf_eigh_batched(const void* M, double* w, void* V, int64_t batch, int64_t nb, void* stream);
/* Replaces _native.eigh_block_sizes (cpp_hf_native.cpp:314-343 ->
 * linalg.hpp:72-120).  sizes is a HOST array of n_sizes positive block sizes. */
int cpphf_eigh_block_sizes(const void* M, double* w, void* V, int64_t batch, int64_t nb,
                           const int64_t* sizes, int64_t n_sizes, int sort, void* stream);
/* Replaces _native.max_offblock_sizes (cpp_hf_native.cpp:345-358 ->
 * linalg.hpp:123-140).  Writes the result to the device scalar *out. */
int cpphf_max_offblock_sizes(const void* M, int64_t batch, int64_t nb, const int64_t* sizes,
                             int64_t n_sizes, double* out, void* stream);

/* ------------------------------------------------------------------------
 * Chemical potential.  Replaces _native.find_mu_bisection
 * (cpp_hf_native.cpp:361-377 -> utils.hpp:49-75) and the in-loop
 * Newton-in-bracket solver of utils.hpp:79-116.  eps (nk, nb) and weights (nk)
 * are device arrays; the result goes to the device scalar *mu_out.  Both run
 * as one cooperative persistent kernel with bounded grid barriers.
 * ---------------------------------------------------------------------- */
size_t cpphf_mu_workspace_bytes(int64_t nk, int64_t nb);
int cpphf_find_mu_bisection(const double* eps, const double* weights, int64_t nk, int64_t nb,
                            double n_e, double T, int maxiter, double* mu_out, void* workspace,
                            size_t workspace_bytes, void* stream);
/* Allocation-free variant of cpphf_find_mu_bisection.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory at call
 * time - a host plug-in whose device memory belongs to a fixed pool it may not
 * grow, or a runtime that forbids cudaMalloc/cudaFree in its critical path
 * because they synchronise the device.  (It makes CUDA calls - it launches a
 * kernel - so like any entry point it must not be called from a host function
 * queued on a stream.)  Same arguments and
 * result as cpphf_find_mu_bisection minus the workspace: the scratch (grid
 * barrier words and block partials, about 74 KB) is a file-scope device array
 * that every GPU loading the library holds until the process exits.  Limit:
 * nk*nb <= CPPHF_MU_NOALLOC_MAX_EIGENVALUES; larger sizes are rejected with
 * CPPHF_ERR_INVALID.  The first call on a device looks up the array's device
 * address (with that device current) and should come before any stream
 * capture; the cached address is not valid across cudaDeviceReset() or a
 * re-created primary context, so do not use this entry point after either.
 * Calls share the array: each call clears the words that must start at zero,
 * and calls that overlap on the GPU race.  Calls no allocating routine. */
#define CPPHF_MU_NOALLOC_MAX_EIGENVALUES 2147483647LL
int cpphf_find_mu_bisection_noalloc(const double* eps, const double* weights, int64_t nk, int64_t nb,
                                    double n_e, double T, int maxiter, double* mu_out, void* stream);
/* mu0 is a device scalar (the warm start). */
int cpphf_solve_mu_inloop(const double* eps, const double* w_norm, int64_t nk, int64_t nb,
                          double n_target_norm, const double* mu0, double T, int maxiter,
                          double* mu_out, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------
 * Kernel view: POD mirror of HFKernel (cpp/include/cpp_hf/kernel.hpp:10-84)
 * with DEVICE pointers.  has_contact is fock.hpp:25-29 evaluated by the caller
 * (any contact_g != 0 or n_contact > 1).  exchange_precision: 64 or 32.
 * ---------------------------------------------------------------------- */
/* Superlattice (moire plane-wave) data of a kernel, mirroring the
 * superlattice_* entries of the reference's kernel_args dict
 * (cpp_hf_native.cpp:109-213, superlattice.py:88-193).  nb = n_G * dim_orb.
 * The CSR pair lists, tile offsets and pair_to_delta are HOST arrays (the
 * channel plan is made on the host every call); the Coulomb tables are device
 * arrays. */
typedef struct cpphf_superlattice {
    int32_t fock_active;     /* streamed superlattice exchange replaces the mesh exchange */
    int32_t hartree_active;  /* superlattice Hartree replaces the diagonal Hartree */
    int64_t n_G, dim_orb, n_delta, N_ext_x, N_ext_y;
    double hartree_degeneracy;
    const void* V_lag_fft;          /* device complex128 (N_ext_x, N_ext_y) */
    const void* V_lag_fft_orbital;  /* device complex128 (N_ext_x, N_ext_y, dim_orb, dim_orb) or NULL */
    const int64_t* g_a_off;         /* host (n_G, 2) */
    const int64_t* pair_i;          /* host (n_pairs) */
    const int64_t* pair_j;          /* host (n_pairs) */
    const int64_t* pair_start;      /* host (n_delta + 1) */
    const int64_t* pair_to_delta;   /* host (n_G, n_G) */
    const double* HH_GG;            /* device (n_G, n_G) or NULL without Hartree */
    const double* HH_GG_orbital;    /* device (n_G, n_G, dim_orb, dim_orb) or NULL */
} cpphf_superlattice;

typedef struct cpphf_kernel {
    int64_t nk1, nk2, nb;
    int64_t dv;
    int32_t include_hartree;
    int32_t include_exchange;
    int32_t exchange_hcp;
    int32_t has_refP;
    int32_t has_contact;
    int32_t n_contact;
    int32_t exchange_precision;
    int32_t hermitian_packing;  /* see below */
    double T;
    double weight_sum;
    const void* h;          /* complex128 (nk1, nk2, nb, nb) */
    const void* VR;         /* complex128 (nk1, nk2, dv, dv) */
    const void* refP;       /* complex128 (nk1, nk2, nb, nb) or NULL */
    const double* w2d;      /* (nk1, nk2) */
    const double* HH;       /* (nb, nb) */
    const double* contact_g;  /* (n_contact) */
    const void* contact_Oi;   /* complex128 (n_contact, nb, nb) */
    const void* contact_Oj;   /* complex128 (n_contact, nb, nb) */
    const cpphf_superlattice* sl;  /* NULL for a plain mesh kernel */
    const void* VR_packed;  /* complex128 packed VR (cpphf_kernel_pack) or NULL */
    const void* h_packed;   /* complex128 packed Hermitian part of h (cpphf_kernel_pack) or NULL */
} cpphf_kernel;

/* Hermitian channel packing (hermitian_packing != 0).  The reference packs the
 * upper triangle of P when V is a real scalar (selfenergy.hpp:119-171, flag
 * exchange_hcp); this extends it to an orbital-resolved V(q) that is
 * Hermitian at every q (VR_ba(R) = conj VR_ab(-R); real symmetric V such as a
 * layer-resolved Coulomb interaction qualifies).  Setting the flag asserts
 * that condition and that every density passed to builds and solves of this
 * kernel is Hermitian (only its upper triangle is read, as in the reference's
 * packed path).  Sigma is then Hermitian, the exchange transforms the
 * nb(nb+1)/2 channels a <= b, and the Fock assembly and energy run inside the
 * last FFT pass.  Applies for nb <= 8, VR of width 1 or nb, no superlattice
 * terms and mesh axes of a supported length; other kernels ignore the flag.
 * VR_packed / h_packed (cpphf_kernel_packed_bytes each) are made once per
 * kernel by cpphf_kernel_pack; when NULL, each build packs them into its
 * workspace (the solvers pack them once per solve).  With the flag set,
 * cpphf_build_fock accepts Sigma == NULL (no Sigma written).  No counterpart in
 * the reference for orbital V. */
size_t cpphf_kernel_packed_bytes(const cpphf_kernel* K);
/* VR_packed (may be NULL; needs dv == nb) and h_packed (may be NULL) of K. */
int cpphf_kernel_pack(const cpphf_kernel* K, void* VR_packed, void* h_packed, void* stream);

/* ------------------------------------------------------------------------
 * Fock build.  Replaces _native.build_fock_apply (cpp_hf_native.cpp:380-415 ->
 * fock.hpp:34-351): Sigma, F = herm(h + Sigma + diag(H) + contact), the
 * k-independent Hartree diagonal hartree_diag (nb) and the energy
 * E = sum_k w_k Re Tr[h P + (Sigma + H)(P - refP)/2] (device scalar *energy).
 * H_dense (complex128 field, may be NULL) receives the dense Hartree term.
 * Sigma may be NULL when K's Hermitian packing applies (see cpphf_kernel).
 * ---------------------------------------------------------------------- */
size_t cpphf_build_fock_workspace_bytes(const cpphf_kernel* K);
int cpphf_build_fock(const cpphf_kernel* K, const void* P, void* Sigma, void* F,
                     double* hartree_diag, double* energy, void* H_dense, void* workspace,
                     size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------
 * Spectral Cayley helpers of the direct-minimisation solver.  Replace
 * _native._cayley_spectral_setup, _cayley_unitary_from_spectrum and
 * _diag_UFU_from_spectrum (cpp_hf_native.cpp:585-651 -> solver_dm.hpp:206-303).
 * ---------------------------------------------------------------------- */
int cpphf_cayley_spectral_setup(const void* d, void* V, double* lam, int64_t batch, int64_t nb,
                                void* stream);
int cpphf_cayley_unitary(const void* V, const double* lam, double tau, void* U, int64_t batch,
                         int64_t nb, void* stream);
int cpphf_diag_ufu(const void* V, const void* Ft_eig, const double* lam, double tau,
                   double* diag, int64_t batch, int64_t nb, void* stream);


/* ------------------------------------------------------------------------
 * Solvers.  The optional projector callback replaces the Python project_fn
 * of the reference (cpp_hf_native.cpp:215-238): it receives a DEVICE field
 * (nk1, nk2, nb, nb) on `stream`, must overwrite it in place before
 * returning, and returns 0 on success.
 * ---------------------------------------------------------------------- */
typedef int (*cpphf_project_fn)(void* user, void* M, int64_t nk1, int64_t nk2, int64_t nb,
                                void* stream);

/* SolverConfig of solver_dm.hpp:22-63 (optimizer 0 = preconditioned CG;
 * block_sizes is a HOST array, validated as the reference does and otherwise
 * ignored: the dense path returns the same density). */
typedef struct cpphf_dm_config {
    int64_t max_iter;
    double tol_E;
    double tol_grad;
    int64_t plateau_window;
    double denom_scale;
    double max_step;
    int64_t cg_restart;
    double bt_shrink;
    int64_t bt_max;
    int32_t mu_maxiter;
    int32_t optimizer;
    const int64_t* block_sizes;
    int64_t n_block_sizes;
    /* Switched precision (no counterpart in the reference): > 0 runs the exchange
     * in complex64 while the Riemannian gradient norm is >= this value, then in
     * complex128 to the end (K->exchange_precision must be 64).  The energy test
     * never ends the solve during the complex64 phase: it switches instead.
     * 0 = plain solve at K->exchange_precision. */
    double mixed_switch_grad;
    /* 1: each iteration's launches are captured once as a CUDA graph and replayed
     * (fewer launch gaps for a single solve); 0: every kernel is launched each
     * iteration (better when many solves share the GPU from several host
     * threads, where per-solve graph instantiation contends in the driver). */
    int32_t graphs;
    /* 1: the projector only enqueues device work on the stream (e.g.
     * cpphf_symmetry_project_fn), so iterations with it may still be captured. */
    int32_t project_device;
    /* optimizer 1, trust-region Newton (SolverConfig.tr_delta0 / tr_cg_max /
     * deflation_* of src/cpp_hf/solver.py:48-59, solver_rtr.hpp:163-205):
     * initial trust radius, Steihaug CG iterations per outer step, and the
     * deflation bias (deflation_targets: device complex128
     * (n_deflation, nk1, nk2, nb, nb) or NULL; off unless n_deflation > 0 and
     * deflation_sigma > 0). */
    double tr_delta0;
    int64_t tr_cg_max;
    const void* deflation_targets;
    int64_t n_deflation;
    double deflation_sigma;
    double deflation_length;
} cpphf_dm_config;

typedef struct cpphf_dm_result {
    double mu;
    double energy;
    int64_t n_iter;
    int32_t converged;
    int32_t reserved;
} cpphf_dm_result;

/* Replaces _native.solve_dm (cpp_hf_native.cpp:488-582 -> solver_dm.hpp:392-653
 * for optimizer 0, solver_rtr.hpp:163-459 for optimizer 1).
 * Q_out, density_out, fock_out (device fields) may be NULL; p_out (device,
 * (nk1, nk2, nb)); hist_E / hist_grad are HOST arrays of max_iter doubles.
 * cpphf_solve_dm_workspace_bytes covers optimizer 0 only; the _cfg form covers
 * the optimizer and deflation settings of *cfg. */
size_t cpphf_solve_dm_workspace_bytes(const cpphf_kernel* K);
size_t cpphf_solve_dm_workspace_bytes_cfg(const cpphf_kernel* K, const cpphf_dm_config* cfg);
int cpphf_solve_dm(const cpphf_kernel* K, const cpphf_dm_config* cfg, const void* P0, double n_e,
                   cpphf_project_fn project, void* project_user, void* Q_out, double* p_out,
                   void* density_out, void* fock_out, double* hist_E, double* hist_grad,
                   cpphf_dm_result* result, void* workspace, size_t workspace_bytes,
                   void* stream);

/* Replaces _native._rtr_joint_hvp (cpp_hf_native.cpp:654-694 ->
 * solver_rtr.hpp:55-111): the joint (Q, p) Hessian-vector product of the
 * trust-region Newton solver, one Fock build of the linear response.  X, Q, Ft,
 * HX: device complex128 (nk1, nk2, nb, nb); dp, p, Hp: device float64
 * (nk1, nk2, nb).  Hp is projected onto sum_k w_k sum_b Hp = 0. */
size_t cpphf_rtr_joint_hvp_workspace_bytes(const cpphf_kernel* K);
int cpphf_rtr_joint_hvp(const cpphf_kernel* K, const void* X, const double* dp, const void* Q, const double* p,
                        const void* Ft, void* HX, double* Hp, void* workspace, size_t workspace_bytes,
                        void* stream);

/* Replaces _native._deflation_bias (cpp_hf_native.cpp:697-716 ->
 * solver_rtr.hpp:124-157): Phi = sigma sum_i exp(-d_i^2 / (2 length^2)) with
 * d_i^2 = sum_k w2d_k |P_k - targets_i,k|_F^2, S_pen = 2 sum_i phi'(d_i^2)
 * (P - targets_i) and diag = 2 sum_i phi'(d_i^2).  P, targets, S_pen: device
 * complex128; w2d: device (nk1, nk2); phi_diag: HOST double[2] <- (Phi, diag).
 * targets NULL, n_deflation 0 or sigma 0 give zeros. */
size_t cpphf_deflation_bias_workspace_bytes(int64_t n_deflation);
int cpphf_deflation_bias(const void* P, const void* targets, int64_t n_deflation, const double* w2d, int64_t nk1,
                         int64_t nk2, int64_t nb, double sigma, double length, void* S_pen, double* phi_diag,
                         void* workspace, size_t workspace_bytes, void* stream);

/* SCFConfig of solver_scf.hpp:20-50; acceleration 0 = linear mixing. */
typedef struct cpphf_scf_config {
    int64_t max_iter;
    double density_tol;
    double comm_tol;
    double mixing;
    double level_shift;
    int32_t acceleration; /* 0 linear mixing, 1 C-DIIS, 2 ODA */
    int32_t reserved;
    /* Switched precision (no counterpart in the reference): > 0 runs the exchange
     * in complex64 until the density residual ||P_new - P||_w and the commutator
     * residual ||[F,P]||_w are both below this value, then in complex128
     * (K->exchange_precision must be 64); convergence is only accepted in the
     * complex128 phase.  0 = plain. */
    double mixed_switch_tol;
    /* acceleration 1 (C-DIIS): history length, first iteration count at which
     * extrapolation starts (at least 2), damping of the extrapolated Fock towards
     * the current one (1 = none); acceleration 2 = ODA (one extra Fock build per
     * iteration).  trust_radius > 0 clips each density step to that weighted
     * norm.  (solver_scf.hpp:200-428, SCFConfig in reference_scf.py:18-57) */
    int32_t diis_size;
    int32_t diis_start;
    double diis_damping;
    double trust_radius;
    /* 1: with linear mixing, no projector and a plain mesh kernel, every
     * iteration after the first (the previous iteration's mix, the Fock build, the
     * occupation step and the residuals) is captured once per precision as a CUDA
     * graph and replayed; 0: every kernel is launched (for many concurrent solves
     * from several host threads). */
    int32_t graphs;
    int32_t reserved1;
    /* block_sizes (HOST array, may be NULL): with more than one block summing to
     * nb, each Fock matrix whose off-block entries are below 1e-10 + 1e-10 of its
     * largest entry is diagonalised block by block (eigenvalues ordered block by
     * block), as density_from_fock does (solver_scf.hpp:96-124).  Disables the
     * per-iteration graph capture (the choice is made on the host). */
    const int64_t* block_sizes;
    int64_t n_block_sizes;
} cpphf_scf_config;

typedef struct cpphf_scf_result {
    double energy;
    double mu;
    int64_t iterations;
    int32_t converged;
    int32_t reserved;
} cpphf_scf_result;

/* Replaces _native.solve_scf (cpp_hf_native.cpp:418-485 -> solver_scf.hpp:156-444).
 * density_out / fock_out device fields (may be NULL); hist_* HOST arrays of
 * max_iter doubles. */
size_t cpphf_solve_scf_workspace_bytes(const cpphf_kernel* K);
/* Workspace of a solve with a given configuration: the DIIS history (2 x
 * diis_size fields and the extrapolated Fock), the ODA trial build (2 fields)
 * and the trust-radius snapshot (1 field) come on top of the linear-mixing
 * size above. */
size_t cpphf_solve_scf_workspace_bytes_cfg(const cpphf_kernel* K, const cpphf_scf_config* cfg);
int cpphf_solve_scf(const cpphf_kernel* K, const cpphf_scf_config* cfg, const void* P0, double n_e,
                    cpphf_project_fn project, void* project_user, void* density_out,
                    void* fock_out, double* hist_E, double* hist_density, double* hist_comm,
                    cpphf_scf_result* result, void* workspace, size_t workspace_bytes,
                    void* stream);

/* Replaces _native.selfenergy_superlattice_streamed (cpp_hf_native.cpp:719-816 ->
 * superlattice.hpp:50-246): per Delta-G channel, the (G_a, G_b) blocks of rho
 * (nkx, nky, n_G, dim_orb, n_G, dim_orb; device) are placed on the extended
 * (N_ext_x, N_ext_y) grid at offsets (nkx, nky) * g_a_off[G_a], convolved with
 * V_lag_fft (or V_lag_fft_orbital per orbital pair) and read back into sigma
 * (same shape, device).  With hermitian_rho a channel whose reversed pairs form
 * another channel fills both (conjugate transpose).  g_a_off, pair_i, pair_j,
 * pair_start are HOST arrays. */
size_t cpphf_superlattice_workspace_bytes(int64_t n_pairs, int64_t n_G, int64_t dim_orb, int64_t N_ext_x,
                                          int64_t N_ext_y, int orbital_vr);
int cpphf_superlattice_streamed(const void* rho, const void* V_lag_fft, const void* V_lag_fft_orbital,
                                const int64_t* g_a_off, const int64_t* pair_i, const int64_t* pair_j,
                                const int64_t* pair_start, int64_t n_delta, int64_t nkx, int64_t nky,
                                int64_t n_G, int64_t dim_orb, int64_t N_ext_x, int64_t N_ext_y,
                                int hermitian_rho, void* sigma, void* workspace, size_t workspace_bytes,
                                void* stream);

/* Replaces density_from_fock (solver_scf.hpp:96-154, dense-eigh branch): eigh of
 * herm(F), mu by bisection on the raw weights (30 iterations), optional level
 * shift, P = herm(V diag(f) V^H).  P, V: device fields; eps (nk, nb) and the
 * scalar mu: device.  The block_sizes fast path is not taken. */
size_t cpphf_density_from_fock_workspace_bytes(int64_t nk, int64_t nb);
int cpphf_density_from_fock(const void* F, const double* w, int64_t nk1, int64_t nk2, int64_t nb,
                            double n_e, double T, double level_shift, void* P, double* eps, void* V,
                            double* mu, void* workspace, size_t workspace_bytes, void* stream);

/* ---- Derivatives (no counterpart in the reference, which has no autograd) ----
 * Gradients follow torch's convention for complex tensors: for a real loss L,
 * grad z = dL/dRe z + i dL/dIm z.  Scalar upstream gradients (gE, gS) are device
 * pointers so that a backward pass needs no host synchronisation. */

/* Adjoint of the exchange map P -> Sigma (cpphf_exchange with refP = NULL, no
 * ifftshift): gP = -IFFT2[FFT2(G) . conj(VR)].  Full channel set (no HCP). */
int cpphf_exchange_adjoint(const void* G, const void* VR, void* gP, int64_t nk1, int64_t nk2,
                           int64_t nb, int64_t dv, void* stream);

/* dL/dVR = -(1/nk) conj(FFT2(P - refP)) . FFT2(G), per channel (dv = nb) or
 * summed over the nb*nb channels (dv = 1).  Workspace: two fields. */
size_t cpphf_exchange_vr_grad_workspace_bytes(int64_t nk1, int64_t nk2, int64_t nb);
int cpphf_exchange_vr_grad(const void* P, const void* refP, const void* G, void* gVR,
                           int64_t nk1, int64_t nk2, int64_t nb, int64_t dv, void* workspace,
                           size_t workspace_bytes, void* stream);

/* Backward of F = herm(h + Sigma + H): gS = gSigma + herm(gF) and gh = herm(gF).
 * gSigma may be NULL; gS or gh may be NULL to skip them. */
int cpphf_fock_backward_prep(const void* gSigma, const void* gF, void* gS, void* gh, int64_t nk,
                             int64_t nb, void* stream);

/* Workspace of the deterministic (last-block) reductions below. */
size_t cpphf_reduce_workspace_bytes(void);

/* E = sum_k w_k Re[Tr(h P) + 1/2 Tr((Sigma + H)(P - refP))] (fock.py:91-107,
 * fock.hpp:324-383) into the device scalar E.  H is a field (H_per_k = 1) or
 * one (nb, nb) matrix shared by all k (H_per_k = 0); Sigma, H, refP may be NULL. */
int cpphf_hf_energy(const void* h, const void* Sigma, const void* H, int H_per_k, const void* P,
                    const void* refP, const double* w, int64_t nk, int64_t nb, double* E,
                    void* workspace, size_t workspace_bytes, void* stream);
/* Gradients of E given the device scalar gE; any output may be NULL.  gH has
 * the shape of H (field or shared (nb, nb)). */
int cpphf_hf_energy_backward(const void* h, const void* Sigma, const void* H, int H_per_k,
                             const void* P, const void* refP, const double* w, const double* gE,
                             int64_t nk, int64_t nb, void* gP, void* gh, void* gSigma, void* gH,
                             void* grefP, void* stream);

/* S = -sum_k w_k sum_i [p ln p + (1 - p) ln(1 - p)], p clipped to [1e-14, 1 - 1e-14]
 * (fock.py:110-115) into the device scalar S; and its gradient dS/dp times gS. */
int cpphf_occupation_entropy(const double* p, const double* w_norm, int64_t nk, int64_t nb,
                             double* S, void* workspace, size_t workspace_bytes, void* stream);
int cpphf_occupation_entropy_backward(const double* p, const double* w_norm, const double* gS,
                                      int64_t nk, int64_t nb, double* gp, void* stream);

/* Vector-Jacobian product of cpphf_density_from_fock (level_shift = 0) with the
 * electron count held fixed: gF = V [D o herm(V^H G V) - diag(w_k f'_i A / Z)] V^H,
 * D_ij = (f_i - f_j)/(eps_i - eps_j), D_ii = f'_i, A = sum Re(G~_ii) f'_i,
 * Z = sum w_k f'_i.  T is the temperature of the occupations f = expit((mu - eps)/T). */
size_t cpphf_density_from_fock_backward_workspace_bytes(void);
int cpphf_density_from_fock_backward(const void* V, const double* eps, const double* mu, double T,
                                     const double* w, const void* G, void* gF, int64_t nk,
                                     int64_t nb, void* workspace, size_t workspace_bytes,
                                     void* stream);

/* Symmetry-averaging projector (cpp_hf src/cpp_hf/symmetry.py:18-117, make_project_fn)
 * on device fields: group average (1/N)(sum_g g A(k) g^H + sum_s s A(-k) s^H)
 * followed by the time-reversal average (A + U conj(A(-k)) U^H)/2.  All arrays
 * are DEVICE complex128: unitary_group (n_unitary, nb, nb) -- pass the identity
 * as a one-element unitary group when only a spatial group is given, as the
 * reference does --, spatial_group (n_spatial, nb, nb), time_reversal_U (nb, nb)
 * or null, scratch one (nk1, nk2, nb, nb) field.  Conventions: 0 "mod" (-i mod
 * n), 1 "flip" (n - 1 - i); axes: bit 0 = axis 0, bit 1 = axis 1.  nb <= 64. */
typedef struct cpphf_symmetry {
    const void* unitary_group;
    int64_t n_unitary;
    const void* spatial_group;
    int64_t n_spatial;
    int32_t spatial_convention;
    int32_t spatial_axes;
    const void* time_reversal_U;
    int32_t tr_convention;
    int32_t tr_axes;
    void* scratch;
} cpphf_symmetry;

/* Projects M in place on `stream`. */
int cpphf_symmetry_project(const cpphf_symmetry* sym, void* M, int64_t nk1, int64_t nk2, int64_t nb, void* stream);
/* The same with the cpphf_project_fn signature (user = const cpphf_symmetry*):
 * pass it as a solver's projector and the solve projects on the device. */
int cpphf_symmetry_project_fn(void* user, void* M, int64_t nk1, int64_t nk2, int64_t nb, void* stream);

/* Replaces _native.resample_kgrid_2d (cpp_hf_native.cpp:819-840 -> utils.hpp:120-176):
 * periodic linear resampling of a complex128 field (nk_old, nk_old, inner) to
 * (nk_new, nk_new, inner) on centred grids (k = 0 at index n/2); device
 * pointers, bitwise the reference's two-pass result. */
int cpphf_resample_kgrid_2d(const void* values, void* out, int64_t nk_old, int64_t nk_new, int64_t inner, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CPPHF_B200_H */
