/*
 * conductor_rigid.h -- C ABI of the B200-native induced-charge conductor solve.
 *
 * This is the drop-in boundary for the hot path of zeesherman/ConductorRigid: the
 * C-style CUDA drivers of cppmodule/ConductorRigid.cuh (gpu_ZeroForce :19-21,
 * gpu_ComputeForce :23-73, MatrixVectorMultiply :76-114, Precondition :117-129) and
 * the parameter derivation of ConductorRigid::SetParams (ConductorRigid.cc:116-379).
 * Plain pointers and sizes only.  Every call returns a cr_status; the reference
 * called exit() on CUDA errors (ConductorRigid.cu:25-33) and on oversize grids
 * (ConductorRigid.cc:181-189) and ignored GMRES non-convergence
 * (ConductorRigid.cu:1142-1147).
 *
 * Conventions:
 *   - N beads indexed 0..N-1 (the reference's active group in index order);
 *     positions are double[N*3] (x,y,z) inside the orthorhombic box [-L/2, L/2).
 *   - B isolated bodies: body[i] is the body tag of bead i (the reference's `body`
 *     list, ConductorRigid.cc:88-95); rigid[b] != 0 for a rigid body (centre
 *     body_pos[b]), 0 for a free bead; body_charge[b] is the known total charge
 *     (the `charge` list, ConductorRigid.cc:98-105).
 *   - Unknowns x = [q (N); Phi (B)], as in the reference's GMRES vector
 *     (ConductorRigid.cu:1118-1128).
 *   - "d_" arguments are device pointers, others host pointers.
 */
#ifndef CONDUCTOR_RIGID_H
#define CONDUCTOR_RIGID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CR_ABI_VERSION 5

typedef enum {
    CR_OK = 0,
    CR_NOT_CONVERGED = 1,   /* iteration limit reached before the tolerance */
    CR_BAD_PARAM = 2,       /* invalid argument or call order */
    CR_CUDA_ERROR = 3,      /* CUDA / cuFFT / kernel launch failure */
    CR_TIMEOUT = 4,         /* a bounded device wait ran out */
    CR_OUT_OF_MEMORY = 5,
    CR_GRID_TOO_LARGE = 6,  /* a grid dimension above 4096 (ConductorRigid.cc:181-189) */
    CR_NOT_READY = 7,       /* topology or positions not set */
    CR_NUMERICAL = 8        /* NaN or Inf in inputs or residuals */
} cr_status;

typedef enum {
    CR_PRECOND_DIAGONAL = 0,  /* the reference's diagonal preconditioner (ConductorRigid.cu:816-859) */
    CR_PRECOND_CONDUCTOR = 1, /* exact isolated-conductor response per body (block inverse) */
    CR_PRECOND_TWO_LEVEL = 2  /* conductor response + a coarse correction on the span of the
                                 bodies' induced dipoles (deflation, built per geometry) */
} cr_preconditioner;

typedef enum {
    CR_FP64 = 0,    /* every operator and reduction in FP64 (the plain solve) */
    CR_MIXED = 1,   /* FP32 operator inside FP64-Arnoldi flexible GMRES, FP64 refinement */
    CR_FP32 = 2     /* FP32 operator only (testing) */
} cr_precision;

/* User parameters.  The first five mirror the Python ConductorRigid(...) keyword
 * arguments (pymodule/compute.py:19: field, xi, errortol); the rest are the
 * overrides the reference hard-codes or derives from errortol. */
typedef struct {
    double field[3];    /* external field E0 (compute.py:19) */
    double xi;          /* Ewald splitting parameter (compute.py:19, default 0.5) */
    double errortol;    /* drives rc, kcut, grid, P (ConductorRigid.cc:123-207) */
    int grid[3];        /* >0 overrides the derived grid (cc:125-178) */
    int support;        /* >0 overrides the derived support P (cc:201) */
    double rcut;        /* >0 overrides rc = sqrt(-ln errortol)/xi (cc:123) */
    double gmres_tol;   /* >0 overrides the GMRES relative tolerance (errortol, cu:1134) */
    int restart;        /* >0 overrides the GMRES restart length (10, cu:1135) */
    int maxiter;        /* >0 overrides the iteration limit (100, cu:1134) */
    int precision;      /* cr_precision */
    int learned;        /* 1: use the learned initial guess / preconditioner correction */
    int precond;        /* cr_preconditioner */
} cr_params;

/* Derived parameters (ConductorRigid.cc:116-207, ConductorRigid.cu:912-917). */
typedef struct {
    int grid[3];
    int support;            /* P after the clamp to the grid (cc:205-207) */
    int support_unclamped;  /* P used for eta (cc:202) */
    double h[3];
    double eta[3];
    double rcut;
    double kcut;
    int n_table;            /* entries - 1 of the real-space tables (cc:279) */
    double dr;              /* table spacing 0.001 (cc:278) */
    double selfcoeff;       /* shell self term (cu:917) */
    double xiterm;          /* 2 xi^2 (cu:915) */
    double prefac;          /* spreading prefactor (cu:916) */
    double quadW;           /* h_x h_y h_z (cu:913) */
} cr_derived;

typedef struct {
    int iterations;           /* Krylov iterations, all levels */
    int restarts;             /* GMRES restart cycles */
    int refinements;          /* outer FP64 refinement steps (CR_MIXED) */
    int matvecs_fp64;
    int matvecs_fp32;
    int converged;            /* 1 when final_residual <= tolerance */
    int used_learned_guess;   /* 1 when the network's initial guess was kept */
    double initial_residual;  /* ||b - A x0|| / ||b|| */
    double final_residual;    /* true FP64 relative residual ||b - A x|| / ||b|| */
    double solve_ms;          /* device time of the solve (CUDA events) */
    double learned_residual;  /* with learned = 1: relative residual of the start after the
                                 guess directions and the potential refit */
    int used_learned_correction;     /* 1 when the learned preconditioner correction was used */
    double correction_reduction[2];  /* one-step residual reduction of the initial residual
                                        without / with the correction (-1: not tried) */
} cr_solve_stats;

typedef struct cr_handle cr_handle;

/* ---- version and errors ---- */
int cr_abi_version(void);
const char *cr_status_string(int status);
/* Message of the last failure on this handle ("" if none). */
const char *cr_last_error(const cr_handle *h);

/* ---- host-only parameter derivation (no GPU needed) ---- */
/* SetParams derivation (ConductorRigid.cc:116-207) for box edges L. */
int cr_derive_params(const cr_params *p, const double L[3], cr_derived *out);
/* Real-space tables (ConductorRigid.cc:278-354): phiq and gradphiq are
 * [n_table+1][2] doubles (.x value at (i+1)*dr, .y the next entry's value). */
int cr_build_tables(const cr_derived *d, double xi, double *phiq, double *gradphiq);

/* ---- lifecycle (ConductorRigid ctor cc:24-106 + SetParams cc:116-379) ---- */
int cr_create(const cr_params *p, const double L[3], cr_handle **out);
int cr_destroy(cr_handle *h);
int cr_get_derived(const cr_handle *h, cr_derived *out);
/* UpdateField (ConductorRigid.cc:382-387). */
int cr_set_field(cr_handle *h, const double field[3]);
/* UpdateParams + SetParams (ConductorRigid.cc:390-400, compute.py:58-60); keeps the
 * topology, rebuilds tables, grid and FFT plans. */
int cr_set_params(cr_handle *h, const cr_params *p, const double L[3]);
/* Body topology (host arrays): body[n_beads], rigid[n_bodies], body_charge[n_bodies]. */
int cr_set_topology(cr_handle *h, int n_beads, const uint32_t *body, int n_bodies,
                    const uint8_t *rigid, const double *body_charge);
/* Stream for all later work on this handle (a cudaStream_t; NULL = legacy default). */
int cr_set_stream(cr_handle *h, void *stream);
/* Captured Arnoldi steps (on by default).  When a stream is set (cr_set_stream, not the
 * legacy default stream) and the profiler is off, a solve captures one Arnoldi step of
 * GMRES (preconditioner, operator, Gram-Schmidt, Hessenberg/Givens update on the
 * device) as a CUDA graph once per geometry and launches it once per iteration, instead
 * of ~25 kernel launches; the iterates are those of the uncaptured loop.  enable = 0
 * keeps every step uncaptured.  cr_graph_launches counts the graph launches. */
/* Mesh tiling of spreading and contraction.  tile_edge T: the mesh is processed in T^3
 * tiles with a (T+P-1)^3 shared-memory halo (T in 2..32, within 227 KB in FP64);
 * spread_mode 0 spreads with per-thread register columns where compiled (T = 8, P = 9
 * or 11), 1 with shared-memory atomics.  cr_set_tiling sets one explicitly; cr_autotune
 * times the FP32 mesh path (spread, FFT, influence function, FFT, contract; reps times)
 * at the given positions for T in {4, 6, 8, 12, 16} and both spread modes where they
 * exist, keeps the fastest and reports it.  Results do not depend on the tiling beyond
 * the summation order of the spreading atomics.  The default is T = 8, mode 0;
 * cr_set_params restores it. */
int cr_set_tiling(cr_handle *h, int tile_edge, int spread_mode);
int cr_autotune(cr_handle *h, const double *d_pos, const double *d_body_pos, int reps, int *tile_edge,
                int *spread_mode, float *best_ms);
int cr_set_graphs(cr_handle *h, int enable);
/* Real-space part of the operator (ConductorRigid.cu:469-567 evaluates the tabulated
 * kernel per neighbour in every product).  Per geometry the in-range bead pairs are
 * found once (32-bead clusters, per cluster pair a 32 x 32 bit mask); the kernel values
 * T(d) of those pairs are then either stored once per geometry and streamed by every
 * product, or evaluated again in every product from the positions (the table in shared
 * memory in FP32).  Stored values are read by one CTA per cluster straight from device
 * memory (the default) or, with CR_REALSPACE_STREAM, streamed through shared memory by
 * bulk copies, one producer warp per CTA.  The real-space product runs concurrently with
 * the wave-space part of the operator (a high-priority side stream of the handle) unless
 * CR_REALSPACE_SERIAL is set or the profiler is on.  flags: CR_REALSPACE_ONFLY32 evaluates the FP32
 * products on the fly, CR_REALSPACE_ONFLY64 the FP64 products (bit-identical to the
 * default stored product); 0 stores both.  Takes effect at the next product. */
#define CR_REALSPACE_ONFLY32 1
#define CR_REALSPACE_ONFLY64 2
#define CR_REALSPACE_STREAM 4
#define CR_REALSPACE_SERIAL 8
int cr_set_realspace(cr_handle *h, int flags);
/* Limit of every bounded device wait of the streamed real-space product
 * (CR_REALSPACE_STREAM), in SM clock
 * cycles (<= 0: the default 2^31, about a second).  A wait that runs out ends the
 * product early; the call that ran it (cr_compute, cr_apply_operator) then returns
 * CR_TIMEOUT and the handle stays usable.  withhold_next != 0 (a test of the waits):
 * the next streamed product issues none of its copies, so its waits run out. */
int cr_set_wait_limit(cr_handle *h, long long cycles, int withhold_next);
int cr_graph_launches(const cr_handle *h, long long *launches);

/* ---- the step (gpu_ComputeForce, ConductorRigid.cu:1153-1286) ----
 * Solves for the bead charges and body potentials (warm start from d_q / d_phi,
 * results written back, as the reference writes HOOMD's charges and
 * m_isolated_potential, cu:1126-1140) and writes bead forces d_force[N*3]
 * (overwritten, as contract_force does, cu:464).  stats may be NULL. */
int cr_compute(cr_handle *h, const double *d_pos, const double *d_body_pos, double *d_q,
               double *d_phi, double *d_force, cr_solve_stats *stats);
/* Same step on host buffers: copies inputs to the device and results back. */
int cr_compute_host(cr_handle *h, const double *pos, const double *body_pos, double *q,
                    double *phi, double *force, cr_solve_stats *stats);

/* ---- operators (for tests and custom solvers) ----
 * cr_set_positions fixes the geometry that the operators below use. */
int cr_set_positions(cr_handle *h, const double *d_pos, const double *d_body_pos);
/* y = A x, x = [q; Phi], y = [Phi_b - M q; sum_b q] (MatrixVectorMultiply,
 * ConductorRigid.cu:953-1020), with the operator in `precision` (CR_FP64/CR_FP32). */
int cr_apply_operator(cr_handle *h, const double *d_x, double *d_y, int precision);
/* The handle's preconditioner: the reference's diagonal scaling (Precondition,
 * ConductorRigid.cu:1023-1044) or the conductor response (cr_params.precond). */
int cr_precondition(cr_handle *h, const double *d_x, double *d_y);
/* Coarse level of CR_PRECOND_TWO_LEVEL for the current positions (built here if the
 * positions changed since): active 1/0, coarse unknowns (three per rigid body of at least
 * four beads), ordered near body pairs, half-space wave vectors of the coarse operator,
 * and 1 when the sparse form (near-pair blocks, CG steps) is in use. */
int cr_coarse_info(cr_handle *h, int *active, int *n_coarse, long long *n_pairs, int *n_modes, int *sparse);
/* Coarse problems with more than max_dense unknowns (default 12288) skip the coarse level
 * (pcg_iterations = 0, the default) or use the sparse form (pcg_iterations > 0): 3 x 3
 * blocks of near body pairs plus the low-rank wave-space term, pcg_iterations
 * block-Jacobi CG steps per application instead of a dense inverse. */
int cr_set_coarse(cr_handle *h, int max_dense, int pcg_iterations);
/* Right-hand side [-(r_i - R_b).E0 ; Q_b] (compute_objective, cu:764-813). */
int cr_objective(cr_handle *h, double *d_rhs);
/* Wave-space potential of charges q (spread, FFT, scale, inverse FFT, contract;
 * ConductorRigid.cu:919-937). */
int cr_wave_potential(cr_handle *h, const double *d_q, double *d_phi, int precision);
/* Spread only: real grid [Nx][Ny][Nz] (spread, ConductorRigid.cu:144-234). */
int cr_spread(cr_handle *h, const double *d_q, double *d_grid, int precision);
/* M q = wave + self + real-space potential (PotentialChargeMultiply without the
 * Phi_b subtraction, ConductorRigid.cu:862-946). */
int cr_apply_M(cr_handle *h, const double *d_q, double *d_Mq, int precision);
/* Electrostatic energy U = 1/2 q.(M q) of bead charges d_q[N] at the positions of the
 * last cr_set_positions / cr_compute (FP64).  Not computed by the reference, whose force
 * pass leaves the energy slot at zero (ConductorRigid.cu:464,661). */
int cr_energy(cr_handle *h, const double *d_q, double *energy);
/* Virial of the electrostatic energy U = 1/2 q.(M q) of bead charges d_q[N] at the
 * positions of the last cr_set_positions / cr_compute (FP64): W_ab = -dU/de_ab under the
 * affine strain r -> (1 + e) r of the bead positions and the box, with the charges and
 * the unit shell radius fixed.  virial[13] (host): [0..5] the real-space tensor
 * 1/2 sum_{i != j} r_ij,a F_ij,b over the real-space pair forces, [6..11] the
 * wave-space tensor (per-mode energies of the spread mesh's spectrum with the strain
 * derivative of the shell kernel j0(k)^2 exp(-k^2/4 xi^2)/k^2), [12] the wave-space
 * energy; components in the order xx, xy, xz, yy, yz, zz.  The external field's term
 * -q_i E0.(r_i - R_b) depends on intra-body vectors only and is not included.  Not
 * computed by the reference, which leaves HOOMD's virial untouched
 * (ConductorRigid.cu:464,661). */
int cr_virial(cr_handle *h, const double *d_q, double *virial);
/* Bead forces for charges q (force pass, ConductorRigid.cu:1256-1278). */
int cr_forces(cr_handle *h, const double *d_q, double *d_force, int precision);
/* Full neighbour list within r_list of the current positions (the pair set of the
 * reference's NeighborListGPUBinned, compute.py:38-44; both directions, no
 * exclusions).  d_count[N], d_head[N]; d_list gets up to `capacity` entries in
 * per-bead ascending order; *total receives the entry count (call once with
 * capacity 0 to size the list). */
int cr_neighbor_list(cr_handle *h, double r_list, int *d_count, int64_t *d_head, int *d_list,
                     int64_t capacity, int64_t *total);

/* ---- instrumentation ----
 * With profiling on, every kernel class below is bracketed by CUDA events on the
 * handle's stream; cr_profile_read returns launches and summed device time of one
 * class since the last reset.  Classes: 0 spread, 1 FFT, 2 influence-function scale,
 * 3 contract, 4 real-space potential, 5 contract force, 6 real-space force,
 * 7 Krylov vector ops, 8 body rows, 9 per-solve geometry (binning, neighbour list),
 * 10 preconditioner. */
int cr_profile(cr_handle *h, int enable);   /* enable/disable; also resets the record */
int cr_profile_read(cr_handle *h, int kernel_class, int *launches, double *total_ms);
/* Sizes of the current per-solve geometry (for traffic and roofline arithmetic). */
typedef struct {
    int64_t real_space_pairs;  /* interacting directed bead pairs of one real-space application */
    int tile_edge;             /* spread/contract tile edge in mesh nodes */
    int n_tiles;               /* mesh tiles */
    int n_beads, n_bodies;
    int64_t cluster_pairs;     /* 32-bead cluster pairs (each with a 128-byte bit mask) */
    int64_t stored_values;     /* value slots stored for them (rows padded per pair) */
} cr_geometry_info;
int cr_get_geometry_info(const cr_handle *h, cr_geometry_info *out);
/* Kernels of this library launched through the handle, and cuFFT executions. */
int cr_counters(const cr_handle *h, long long *kernel_launches, long long *fft_execs);

/* ---- rigid-body dynamics ----
 * No counterpart in the reference, which leaves time integration to HOOMD's rigid-body
 * integrator.  cr_body_force_torque sums bead forces d_force[N*3] (from cr_compute)
 * into body forces d_body_force[B*3] and torques d_body_torque[B*3] about the body
 * centres d_body_pos[B*3] (minimum-image bead offsets, FP64).
 * cr_brownian_step takes one overdamped Brownian step of every body in place:
 * translation mu_t F dt + sqrt(2 kT mu_t dt) g, mu_t = 1/(6 pi viscosity a_b);
 * rotation (rigid bodies only) by the angle vector mu_r T dt + sqrt(2 kT mu_r dt) g',
 * mu_r = 1/(8 pi viscosity a_b^3), about the body centre; d_radius[B] holds a_b.  Bead
 * and body positions are wrapped into [-L/2, L/2).  The Gaussian numbers g, g' are a
 * pure function of (seed, step, body): SplitMix64 counters and the Box-Muller
 * transform, so a trajectory does not depend on launch shape or device.  The steric
 * repulsion is added to the body forces (all pairs, minimum image). */
typedef struct {
    double dt;          /* time step */
    double kT;          /* thermal energy */
    double viscosity;   /* solvent viscosity */
    uint64_t seed;      /* noise stream */
    double repulsion;   /* stiffness k of the steric body-body repulsion (0: none): a pair
                           whose centre distance d is below a_i + a_j + contact_gap is pushed
                           apart along the centre line by k (a_i + a_j + contact_gap - d) */
    double contact_gap; /* surface gap at which the repulsion starts */
} cr_brownian_params;
int cr_body_force_torque(cr_handle *h, const double *d_pos, const double *d_body_pos, const double *d_force,
                         double *d_body_force, double *d_body_torque);
int cr_brownian_step(cr_handle *h, const cr_brownian_params *p, int64_t step, const double *d_radius,
                     const double *d_force, double *d_pos, double *d_body_pos);

/* ---- the learned initial guess: per-bead network on the tensor cores ----
 * No counterpart in the reference.  A 48 -> 128 -> 128 -> 1 GELU network with BF16
 * operands and FP32 accumulation on the sm_100 tensor cores (tcgen05, accumulators in
 * tensor memory).  Parameters are one FP32 vector of CR_MLP_PARAMS values:
 * W1[128][48], b1[128], W2[128][128], b2[128], w3[128], b3.  Features are BF16 rows of
 * 48 values (16-byte aligned).  cr_mlp_forward writes y[n]; cr_mlp_accumulate_grad adds
 * the gradient of (1/n) sum (y - t)^2 to the network's gradient buffer and returns the
 * loss; cr_mlp_adam applies one Adam step (gradients clipped to +-clip) and clears the
 * buffer.  Device waits are bounded: a wait that runs out returns CR_TIMEOUT.
 * Needs an sm_100 GPU (CR_BAD_PARAM otherwise). */
#define CR_MLP_FEATURES 48
#define CR_MLP_HIDDEN 128
#define CR_MLP_PARAMS 22913
typedef struct cr_mlp cr_mlp;
int cr_mlp_create(uint64_t seed, cr_mlp **out);
int cr_mlp_destroy(cr_mlp *net);
const char *cr_mlp_last_error(const cr_mlp *net);
int cr_mlp_get_params(cr_mlp *net, float *params);
int cr_mlp_set_params(cr_mlp *net, const float *params);
int cr_mlp_get_grads(cr_mlp *net, float *grads);
int cr_mlp_forward(cr_mlp *net, int n, const uint16_t *d_x, float *d_y, void *stream);
int cr_mlp_accumulate_grad(cr_mlp *net, int n, const uint16_t *d_x, const float *d_t, double *loss, void *stream);
int cr_mlp_adam(cr_mlp *net, double lr, double clip, void *stream);
int cr_mlp_counters(const cr_mlp *net, long long *kernel_launches, long long *adam_steps);
/* Failure detection of the bounded waits.  max_cycles: the clock-cycle limit of every
 * wait of the network's kernels on a tensor-core barrier (default 2^31, about a second
 * at 2 GHz; at least 1000).  withhold_next != 0 makes the next forward or training
 * launch issue neither the first tile's MMAs nor their commit in every CTA, so nothing
 * arrives on the barrier: each CTA's wait runs out, the CTA frees its tensor memory and
 * exits, and the call returns CR_TIMEOUT; the network stays usable (a test hook for the
 * timeout path: nothing faults or hangs, no tensor-core work is left in flight). */
int cr_mlp_set_wait(cr_mlp *net, long long max_cycles, int withhold_next);

/* ---- learned guess for time stepping ----
 * No counterpart in the reference (its solve starts from the previous step's charges,
 * ConductorRigid.cu:1118-1128).  With cr_params.learned = 1 a solve first (1) adds to
 * its start x0 the combination sum_j c_j D_j of the directions D set by
 * cr_set_guess_directions that minimises ||b - A x0|| (one operator application per
 * direction, FP32 in CR_MIXED, then the FP64 residual; a direction that does not help
 * gets c_j = 0), then (2) refits every body potential to the mean of its bead residuals
 * (exact, no operator application), and runs the usual solve from there.
 * cr_solve_stats reports the residual this start reaches and whether it lowered the
 * initial one.  Directions are [n_dir][N+B] device vectors, used by the next solve
 * only; passing the previous solution as one of them keeps both it and the zero vector
 * in reach, so the start is never worse than either.
 * The helpers build the two directions of the learned guess between time steps from the
 * previous solution q' at positions (r', R') and the new positions (r, R):
 *   cr_bead_neighbors   the CR_GUESS_BEAD_NEIGHBORS nearest same-body beads of each bead;
 *   cr_body_neighbors   the CR_GUESS_BODY_NEIGHBORS nearest bodies of each body (centres);
 *   cr_guess_features   FP32 features [N][CR_MLP_FEATURES] and the transport term
 *                       s_i = grad_s q'(r'_i) . (rotation displacement of bead i);
 *   cr_feature_stats    per-feature sums and sums of squares [2][48] (FP64);
 *   cr_feature_pack     standardised BF16 rows for the network;
 *   cr_guess_target     network target (q - q') / scale;
 *   cr_neutral_direction scale * v minus per-body means (charge rows unchanged), Phi 0. */
#define CR_GUESS_BEAD_NEIGHBORS 6
#define CR_GUESS_BODY_NEIGHBORS 8
#define CR_MAX_GUESS_DIRECTIONS 4
int cr_set_guess_directions(cr_handle *h, int n_dir, const double *d_dirs);
int cr_bead_neighbors(cr_handle *h, const double *d_pos, int *d_nbr);
int cr_body_neighbors(cr_handle *h, const double *d_body_pos, int *d_nbr);
int cr_guess_features(cr_handle *h, const double *d_radius, const int *d_bead_nbr, const int *d_body_nbr,
                      const double *d_q_prev, const double *d_pos_prev, const double *d_body_pos_prev,
                      const double *d_pos, const double *d_body_pos, float *d_feat, double *d_transport);
int cr_feature_stats(cr_handle *h, int n, const float *d_feat, double *d_sums);
int cr_feature_pack(cr_handle *h, int n, const float *d_feat, const float *d_mu, const float *d_inv_sigma,
                    uint16_t *d_x);
int cr_guess_target(cr_handle *h, const double *d_q, const double *d_q_prev, double scale, float *d_t);
int cr_neutral_direction(cr_handle *h, const void *d_v, int v_is_fp32, double scale, double *d_dir);

/* ---- the learned correction of the preconditioner ----
 * No counterpart in the reference, whose GMRES applies the fixed diagonal scaling of
 * Precondition (ConductorRigid.cu:1023-1044) to every Krylov vector.  With a network set,
 * every flexible-GMRES step of a solve preconditions its Krylov vector v with
 * z' = P v + weight * s * y, P the handle's preconditioner, s the RMS of P v and y the
 * network's per-bead output for 48 features of (v, P v) (the vectors at unit RMS, the own
 * body's mean and induced dipole of P v, the field direction, and for the 8 nearest bodies
 * their direction, proximity, mean of P v and the potential of their induced dipole).
 * Before a solve uses it, the correction c of the solve's initial residual r is tried:
 * it is used only if the least-squares residual of r over span{A P r, A c} is at least
 * 1 % below the one over span{A P r} alone, and then at the scale that fit gives it (z' = P v +
 * (a_c / a_p) weight s y); otherwise the solve falls back to the plain preconditioner.
 * cr_solve_stats reports the choice and both relative residuals.  The network is the caller's
 * (cr_mlp_create); net = NULL removes it, weight = 0 keeps it set without applying it.
 * Flexible GMRES keeps the fixed point and the true-residual stopping test whatever the
 * network outputs.
 * cr_correction_samples writes training rows from the last solve on this handle: for up
 * to max_dirs stored preconditioned Krylov directions z_j of its last cycle, the features
 * of (w, P w), w = A z_j (FP64), into d_x [rows][48] (BF16, 16-byte aligned) and the
 * targets (z_j - P w) / s into d_t [rows]; *rows = directions used x N.  Train the network
 * on them with cr_mlp_accumulate_grad / cr_mlp_adam. */
int cr_set_correction(cr_handle *h, cr_mlp *net, double weight);
int cr_correction_samples(cr_handle *h, int max_dirs, uint16_t *d_x, float *d_t, int *rows);

/* ---- batched independent systems ----
 * No counterpart in the reference (one system per force compute).  Solves n independent
 * systems, each through its own handle (its own parameters, box, mesh and topology), as
 * cr_compute would one by one, but side by side: a pool of n_threads host threads
 * (<= 0: 16), each with its own non-blocking stream, takes the systems largest first.
 * status[i] receives each cr_compute status, stats (may be NULL) each solve's
 * statistics; the return value is the worst status.  Each handle's own stream setting
 * is restored afterwards.  Call every handle once with cr_compute before batching: its
 * first solve allocates device memory, which synchronises the device. */
int cr_batch_compute(int n, cr_handle *const *handles, const double *const *d_pos, const double *const *d_body_pos,
                     double *const *d_q, double *const *d_phi, double *const *d_force, cr_solve_stats *stats,
                     int *status, int n_threads);

/* ---- lockstep batches: all replicas advanced together, one launch per stage ----
 * No single counterpart in the reference, which solves one system per computeForces
 * (ConductorRigid.cu:1153-1286); each replica is solved by that path
 * (MatrixVectorSolve, ConductorRigid.cu:1051-1151, with the operator of
 * ConductorRigid.cu:862-1020).
 *
 * cr_batch_create groups n existing handles (each with its topology set) into a batch
 * whose solves advance every unconverged replica by one Arnoldi step per round, each
 * stage of the step (preconditioner, charge cast, spreading, the transforms of each mesh
 * size, influence function, contraction, real-space product, rows, body sums,
 * Gram-Schmidt, Givens rotations) one kernel launch over all replicas.  The members must
 * share the precision (CR_MIXED or CR_FP64), preconditioner, restart length and support
 * (9 or 11), use 8^3 mesh tiles with register-column spreading (the default tiling),
 * stored real-space values with the direct product, and no learned start or correction;
 * cr_batch_create returns CR_BAD_PARAM otherwise (message from cr_batch_last_error(NULL)
 * on the calling thread).  The batch keeps each replica's mesh size, box and influence
 * function as they were at creation: after cr_set_params on a member, make a new batch.
 * The handles stay owned by the caller and must outlive the batch; do not use them
 * concurrently with cr_batch_solve. */
typedef struct cr_batch cr_batch;
int cr_batch_create(int n, cr_handle *const *handles, cr_batch **out);
int cr_batch_destroy(cr_batch *batch);
const char *cr_batch_last_error(const cr_batch *batch);
/* Solve every replica (arguments as cr_batch_compute: per-replica device arrays; d_q and
 * d_phi hold the start and receive the solution, d_force the forces).  Per-geometry work
 * (geometry, stored values, coarse level) and the FP64 force pass run per replica as tasks
 * of n_threads host threads (<= 0: 16) with one stream each, largest replicas first; a
 * replica joins the lockstep rounds (on the batch's own streams) as soon as its set-up is
 * done and leaves for its force pass as soon as it has converged, so set-up, iterations
 * and forces of different replicas overlap on the GPU.  status[i] receives each replica's status, stats (may be
 * NULL) its statistics (solve_ms: the lockstep loop, the same for all replicas); the
 * return value is the worst status. */
int cr_batch_solve(cr_batch *batch, const double *const *d_pos, const double *const *d_body_pos,
                   double *const *d_q, double *const *d_phi, double *const *d_force, cr_solve_stats *stats,
                   int *status, int n_threads);
/* Batched kernel launches, batched transforms and lockstep rounds since creation. */
int cr_batch_counters(const cr_batch *batch, long long *kernel_launches, long long *fft_execs, long long *steps);
/* Timings of the last cr_batch_solve: host-clock ms until the first replica finished its
 * set-up and joined the rounds, device ms from then to the end (CUDA events on the
 * batch's stream), host-clock ms of the whole call. */
int cr_batch_phase_ms(const cr_batch *batch, double *first_join_ms, double *rounds_ms, double *total_ms);

/* ---- spreading without device allocation ----
 * No counterpart in the reference.  For callers that cannot allocate device memory
 * where they need the charge mesh: a host engine that owns all device memory through
 * its own pool, or a time-step loop in which cudaMalloc/cudaFree would synchronise the
 * device while other streams run.  Same result as cr_spread in FP64 (ConductorRigid.cu
 * spreading rule) for derived parameters d (from cr_derive_params / cr_get_derived),
 * Ewald parameter xi and box L; device arrays d_pos[n_beads*3], d_q[n_beads] in,
 * d_grid[Nx*Ny*Nz] out (overwritten).  It allocates nothing: its scratch is one
 * file-scope device array of CR_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library holds until exit, located per device with cudaGetSymbolAddress on the first
 * call on that device (make that first call before any stream capture).  The address
 * is kept for the life of the process: after cudaDeviceReset on a device, do not call
 * this entry point on that device again.  At most CR_NOALLOC_MAX_BEADS beads,
 * CR_NOALLOC_MAX_TILES 8^3-node mesh tiles and support 16; larger inputs are rejected
 * with CR_BAD_PARAM and a message in cr_noalloc_last_error().  All calls share the
 * array, so calls that overlap on the GPU race and must be serialised by the caller.
 * Every call reads a position-check flag back to the host after its first kernel and
 * waits for the end of its work on `stream` before returning, so each call blocks the
 * calling thread until its spreading has finished. */
#define CR_NOALLOC_MAX_BEADS 262144
#define CR_NOALLOC_MAX_TILES 32768
#define CR_NOALLOC_SCRATCH_BYTES 6291456
int cr_spread_noalloc(const cr_derived *d, double xi, const double L[3], int n_beads, const double *d_pos,
                      const double *d_q, double *d_grid, void *stream);
/* Message of the last cr_spread_noalloc failure on the calling thread ("" if none). */
const char *cr_noalloc_last_error(void);

/* ---- synthetic systems (host utilities for the benchmark workloads) ---- */
int cr_util_icosphere_count(int level);
int cr_util_icosphere(int level, double *verts);
int cr_util_place_spheres(int n, const double *radii, const double L[3], uint64_t seed,
                          int64_t max_attempts, double *centres);
int cr_util_uniform(uint64_t seed, int64_t n, double *out);

#ifdef __cplusplus
}
#endif
#endif /* CONDUCTOR_RIGID_H */
