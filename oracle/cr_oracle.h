/*
 * cr_oracle.h -- FP64 CPU restatement of ConductorRigid's induced-charge solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product in
 * conductorrigid_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  Nothing in the product links or calls it.
 *
 * Parity status: parity unpinned against reference outputs.  The reference
 * (HOOMD-blue 1.x plugin, cppmodule/ConductorRigid.{cc,cu}) needs HOOMD, CUSP and
 * Boost, none of which exist here, and its kernels use CUDA texture references that
 * CUDA 12 removed, so it cannot be built or run and ships no golden vectors or
 * tests.  The restatement is instead pinned by known-answer tests in tests/
 * (classic Ewald k-sum, Ewald-split independence, free-space dense solve of an
 * isolated conductor, finite-difference energy derivative of the forces, exact
 * charge constraints, an independent NumPy restatement of the parameter and
 * table derivation).
 *
 * Every function cites the reference file:line it follows.  All arithmetic is
 * IEEE double.  Conventions shared with the product:
 *   - beads are indexed 0..N-1 ("group order": the reference indexes the GMRES
 *     vector by active-group index and reads charges by global index, which only
 *     agree when group == all particles in index order, ConductorRigid.cu:994,169);
 *   - body[i] is the isolated-body tag of bead i (ConductorRigid.cc:88-95);
 *   - rigid[b] != 0 marks a rigid body (centre body_pos[b], preconditioner 1/size),
 *     rigid[b] == 0 a free bead (preconditioner 1/(4 pi), zero objective);
 *   - the box is orthorhombic with its origin at -L/2 (HOOMD BoxDim).
 */
#ifndef CR_ORACLE_H
#define CR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Inputs and derived parameters of SetParams (ConductorRigid.cc:116-207). */
typedef struct {
    /* inputs */
    double L[3];          /* box edge lengths */
    double xi;            /* Ewald splitting parameter */
    double errortol;      /* error tolerance that drives the derivation */
    int grid_override[3]; /* >0: use this grid size instead of the derived one */
    int support_override; /* >0: use this P instead of the derived one */
    double rc_override;   /* >0: use this real-space cutoff */
    /* derived */
    int N[3];             /* grid nodes per dimension */
    int P;                /* support (clamped to the grid) */
    int P_unclamped;      /* support used for eta (cc:202 runs before the clamp) */
    double h[3];          /* grid spacing */
    double eta[3];        /* spectral splitting parameter */
    double rc;            /* real-space cutoff */
    double kcut;          /* wave-space cutoff */
    int N_table;          /* real-space table entries - 1 */
    double dr;            /* table spacing */
    double selfcoeff;     /* shell self term (cu:917) */
    double xiterm;        /* 2 xi^2 (cu:915) */
    double prefac;        /* spreading prefactor (cu:916) */
    double quadW;         /* h_x h_y h_z (cu:913) */
} orc_params;

/* Error codes. */
enum { ORC_OK = 0, ORC_GRID_TOO_LARGE = 1, ORC_BAD_INPUT = 2, ORC_RC_TOO_LARGE = 3 };

int orc_derive(orc_params *p);
/* Real-space tables, [N_table+1][2] doubles each (.x value, .y next value). */
void orc_tables(const orc_params *p, double *phiq, double *gradphiq);
/* Wave-space scale on the full grid [Nx][Ny][Nz] (cc:245-274). */
void orc_scale(const orc_params *p, double *scale);

/* In-place complex 3D DFT of re/im [n0][n1][n2]; sign -1 forward, +1 inverse,
 * unnormalised (cuFFT conventions). */
void orc_fft3d(int n0, int n1, int n2, double *re, double *im, int sign);

/* Spread charges onto a real grid [Nx][Ny][Nz] (ConductorRigid.cu:144-234). */
void orc_spread(const orc_params *p, int N, const double *pos, const double *q, double *grid);
/* Contract a real grid to bead potentials (cu:260-360). */
void orc_contract(const orc_params *p, int N, const double *pos, const double *grid, double *phi);
/* Contract a real grid to bead forces, overwrite (cu:363-466). */
void orc_contract_force(const orc_params *p, int N, const double *pos, const double *q,
                        const double *grid, double *force);
/* Wave-space potential: spread, FFT, scale, inverse FFT, contract (cu:919-937). */
void orc_wave_potential(const orc_params *p, int N, const double *pos, const double *q, double *phi);
/* Wave-space force (cu:1256-1274). */
void orc_wave_force(const orc_params *p, int N, const double *pos, const double *q, double *force);

/* Full neighbour list within r_list (all j != i, minimum image, both directions,
 * sorted by j).  Two calls: with list == NULL it fills count[] and returns the total;
 * then with head/list it fills them.  Distances use dx -= L*rint(dx*(1/L)) and
 * d2 = dx*dx + dy*dy + dz*dz without fused multiply-add. */
int64_t orc_neighbor_list(int N, const double *pos, const double L[3], double r_list,
                          int *count, int64_t *head, int *list);

/* Real-space potential plus self term over a neighbour list (cu:469-567):
 * phi_io enters holding the wave-space part and leaves holding phi total (M q). */
void orc_real_space(const orc_params *p, int N, const double *pos, const double *q,
                    const double *phiq_table, const int64_t *head, const int *count,
                    const int *list, double *phi_io);
/* Real-space force (cu:570-664): force_io += q_i E0 + sum_j -T'(d) q_i q_j rhat. */
void orc_real_space_force(const orc_params *p, int N, const double *pos, const double *q,
                          const double E0[3], const double *gradphiq_table,
                          const int64_t *head, const int *count, const int *list,
                          double *force_io);

/* Opaque solver context: parameters, tables, scale, topology, neighbour list. */
typedef struct orc_ctx orc_ctx;
orc_ctx *orc_create(const orc_params *p, int N, int B, const uint32_t *body,
                    const uint8_t *rigid, const double *body_charge);
void orc_destroy(orc_ctx *c);
/* Set positions (N*3) and body centres (B*3); builds the neighbour list. */
int orc_set_positions(orc_ctx *c, const double *pos, const double *body_pos);
/* M q: wave + self + real (no potential subtraction). */
void orc_apply_M(orc_ctx *c, const double *q, double *Mq);
/* y = A x with x = [q; Phi], y = [Phi_b - M q; sum_b q] (cu:953-1020). */
void orc_matvec(orc_ctx *c, const double *x, double *y);
/* Diagonal preconditioner (cu:816-859, rigid rows 1/size, free rows 1/(4 pi)). */
void orc_precondition(orc_ctx *c, const double *x, double *y);
/* Right-hand side [-(r_i - R_b).E0 ; Q_b] (cu:764-813). */
void orc_objective(orc_ctx *c, const double E0[3], double *rhs);
/* Restarted GMRES with the semantics of the reference's cusp::krylov::gmres call
 * (cu:1134-1136): left preconditioned, restart R, stop when the preconditioned
 * residual norm <= tol * ||b|| or after maxiter iterations.  x is the warm start.
 * Returns the iteration count; *resid gets the final preconditioned residual
 * estimate and *true_rel the true relative residual ||b - A x|| / ||b||. */
int orc_gmres(orc_ctx *c, double *x, const double *b, int restart, int maxiter, double tol,
              double *resid, double *true_rel);
/* Bead forces for charges q (cu:1256-1278). */
void orc_forces(orc_ctx *c, const double *q, const double E0[3], double *force);
/* Whole step: objective, GMRES from the warm start (q_io, phi_io), forces. */
int orc_solve(orc_ctx *c, const double E0[3], double *q_io, double *phi_io, double *force,
              int restart, int maxiter, double tol, double *true_rel);
int orc_num_threads(void);

/* Synthetic systems (cr_systems.cc): icosphere vertices, SplitMix64 uniforms and
 * random sequential addition of non-overlapping spheres in a periodic box. */
int orc_icosphere_count(int level);
int orc_icosphere(int level, double *verts);
int orc_uniform(uint64_t seed, int64_t n, double *out);
int orc_place_spheres(int n, const double *radii, const double L[3], uint64_t seed, int64_t max_attempts,
                      double *centres);

#ifdef __cplusplus
}
#endif
#endif
