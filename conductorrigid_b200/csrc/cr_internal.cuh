// cr_internal.cuh -- internal types of the CUDA implementation behind conductor_rigid.h.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/conductor_rigid.h"

namespace cr {

constexpr double kPi = 3.14159265358979323846;

// ---- precision traits ----
template <typename R> struct Prec;
template <> struct Prec<float> {
    typedef float4 R4;
    typedef float2 R2;
    typedef cufftComplex C;
    static constexpr cufftType kR2C = CUFFT_R2C;
    static constexpr cufftType kC2R = CUFFT_C2R;
};
template <> struct Prec<double> {
    typedef double4 R4;
    typedef double2 R2;
    typedef cufftDoubleComplex C;
    static constexpr cufftType kR2C = CUFFT_D2Z;
    static constexpr cufftType kC2R = CUFFT_Z2D;
};

inline cufftResult fft_forward(cufftHandle p, float *in, cufftComplex *out) { return cufftExecR2C(p, in, out); }
inline cufftResult fft_forward(cufftHandle p, double *in, cufftDoubleComplex *out) { return cufftExecD2Z(p, in, out); }
inline cufftResult fft_inverse(cufftHandle p, cufftComplex *in, float *out) { return cufftExecC2R(p, in, out); }
inline cufftResult fft_inverse(cufftHandle p, cufftDoubleComplex *in, double *out) { return cufftExecZ2D(p, in, out); }

// Device buffers of one operator precision.
template <typename R> struct MeshBuffers {
    typedef typename Prec<R>::R4 R4;
    typedef typename Prec<R>::R2 R2;
    typedef typename Prec<R>::C C;
    R4 *pos = nullptr;          // [N] bead positions in the box (x, y, z, 0)
    R2 *phiq = nullptr;         // [n_table+1] potential table (value, next value)
    R2 *gradphiq = nullptr;     // [n_table+1] gradient table
    R *grid = nullptr;          // [Nx*Ny*Nz] real mesh
    C *spec = nullptr;          // [Nx*Ny*(Nz/2+1)] half spectrum
    R *scale = nullptr;         // [Nx*Ny*(Nz/2+1)] influence function S(k)/Ngrid
    R *q = nullptr;             // [N] charges in this precision
    R *phi = nullptr;           // [N] wave-space potential scratch
    R *force = nullptr;         // [3N] wave-space force scratch
    cufftHandle plan_fwd = 0, plan_inv = 0;
    bool ready = false;
};

// Geometry of the current positions (fixed during one solve).
struct Geometry {
    int4 *wstart = nullptr;     // [N] first window node per dim (wrapped), .w = tile id
    int *tile_start = nullptr;  // [ntiles+1]
    int *tile_beads = nullptr;  // [N] beads sorted by tile (ascending bead index within a tile)
    int *tile_count = nullptr;  // [ntiles]
    // neighbour list within rc (CSR; per-bead ascending order)
    int *nl_count = nullptr;    // [N]
    int64_t *nl_head = nullptr; // [N]
    int *nl_list = nullptr;     // [capacity]
    int64_t nl_capacity = 0;
    int64_t nl_total = 0;
    // cell list used to build it
    int *cell_of = nullptr;     // [N]
    int *cell_start = nullptr;  // [ncell+1]
    int *cell_beads = nullptr;  // [N]
    int ncell[3] = {0, 0, 0};
    size_t ncell_alloc = 0;
    bool valid = false;
};

// Real-space operator of the current geometry: 32-bead clusters, cluster pairs
// (I <= J) within rc, per pair a 32x32 bit mask and the packed kernel values.
struct RealSpace {
    int nclus = 0;
    int *sorted = nullptr;          // [N] beads in Morton order
    int *members = nullptr;         // [nclus*32] bead index or -1
    double4 *centre = nullptr;      // [nclus]
    double4 *extent = nullptr;      // [nclus] half extents
    int *count = nullptr;           // [nclus] pairs owned by cluster I
    long long *head = nullptr;      // [nclus] first pair of cluster I
    int *pair_i = nullptr, *pair_j = nullptr;
    long long npairs = 0, pair_cap = 0;
    unsigned *masks = nullptr;      // [npairs*32] row bit masks of in-range bead pairs
    int *nnz_pair = nullptr;        // [npairs] set bits per pair
    long long *voff = nullptr;      // [npairs] first packed value of each pair
    long long nnz = 0;              // stored value slots (rows padded to each pair's longest row)
    long long npairs_beads = 0;     // interacting directed bead pairs (set mask bits)
    unsigned long long *bits = nullptr;
    float *vals32 = nullptr;        // [nnz] packed T(d) values
    double *vals64 = nullptr;
    long long blocks32_cap = 0, blocks64_cap = 0;
    bool valid32 = false, valid64 = false;
    float *acc32 = nullptr;         // [nclus*32] charges in cluster order
    double *acc64 = nullptr;
    float *ysum32 = nullptr;        // [nclus*32] sums of the streamed product (cleared after use)
    double *ysum64 = nullptr;
    double *freal = nullptr;        // [3N] real-space forces
    float4 *boff = nullptr;         // [nclus*32] bead offsets from their cluster centre (FP32)
    float4 *pshift = nullptr;       // [npairs] centre offset of the pair (minimum image), .w = 1 when
                                    // bead separations need no further image
    // streamed product (one per operator precision): the CTAs' cluster ranges and chunks
    struct StreamPlan {
        int ctas = 0;
        int *cl0 = nullptr;             // [ctas+1] first cluster of each CTA
        long long *cbase = nullptr;     // [ctas+1] first chunk of each CTA
        long long *cstart = nullptr;    // [chunks] absolute first byte of each chunk
        long long cap = 0;              // capacity of cstart
        bool valid = false;
    };
    StreamPlan plan32, plan64;
    int *err = nullptr;             // device error word of the streamed product (1: a wait ran out)
    long long wait_limit = 1LL << 31;  // cycles of one bounded wait (about a second)
    int withhold_next = 0;          // the next streamed product issues no copies (test of the waits)
};

// Learned correction of the preconditioner (correction.cu).
struct Correction {
    cr_mlp *net = nullptr;              // the caller's network (not owned); null: no correction
    double weight = 1.0;
    double scale = 1.0;                 // fitted scale of the correction in the current solve
    int active = 0;                     // used by the current solve (decided per solve)
    double last_rho[2] = {-1.0, -1.0};  // one-step residual reduction without / with it
    uint16_t *x = nullptr;              // [N][48] BF16 feature rows
    float *y = nullptr;                 // [N] network output
    int *nbr = nullptr;                 // [B][8] nearest bodies
    double4 *mom = nullptr;             // [B] mean and induced dipole of the preconditioned vector
    double *ss = nullptr;               // [2] squared norms of z and v
    double *zp = nullptr, *zc = nullptr;  // [N+B] scratch
    int cap_n = -1, cap_b = -1;
    long long nbr_gen = -1;
};

// GMRES workspace (FP64).
struct Krylov {
    int n = 0, m = 0;
    double *V = nullptr;        // [(m+1) * n] orthonormal basis
    double *Z = nullptr;        // [m * n] preconditioned directions (flexible GMRES)
    double *w = nullptr;        // [n]
    double *r = nullptr;        // [n]
    double *b = nullptr;        // [n]
    double *x = nullptr;        // [n]
    double *d = nullptr;        // [n] refinement correction
    double *rr = nullptr;       // [n] refinement residual (right-hand side of the inner solve)
    double *partial = nullptr;  // [nblocks * (m+2)] dot-product partials
    double *hcol = nullptr;     // [m+2] reduced dot products
    double *yvec = nullptr;     // [m] least-squares coefficients
    double *h_pinned = nullptr; // pinned host mirror of hcol
    int nblocks = 0;
    int last_cols = 0;          // Z columns filled by the last cycle
    // captured Arnoldi step (CUDA graph): device-side Hessenberg bookkeeping
    double *H = nullptr;        // [(m+1) * m] row-major Hessenberg, rotated in place
    double *cs = nullptr, *sn = nullptr;  // [m] Givens rotations
    double *g = nullptr;        // [m+1] rotated right-hand side
    double *sin = nullptr, *sz = nullptr; // [n] staging of V_j and Z_j (fixed addresses for the graph)
    int *state = nullptr;       // device ArnoldiState
    void *h_state = nullptr;    // pinned mirror of ArnoldiState
    double *h_hg = nullptr;     // pinned [(m+1)*m + (m+1)]: H and g at the end of a cycle
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // per operator precision (FP64, FP32)
    long long exec_gen[2] = {-1, -1};              // geometry generation captured
    int exec_corr[2] = {0, 0};                     // learned correction inside the captured step
    long long exec_kernels[2] = {0, 0}, exec_ffts[2] = {0, 0};  // work per launch
};

// Conductor-response preconditioner: one K^-1 per distinct body shape.
struct ConductorPrecond {
    bool ready = false;
    int n_shapes = 0, max_n = 0;
    int *d_body_shape = nullptr;        // [B]
    int *d_shape_n = nullptr;           // [S] beads per shape
    long long *d_shape_mat = nullptr;   // [S] offset of the shape's K^-1 (column-major n x n)
    int *d_shape_vec = nullptr;         // [S] offset of the shape's u = K^-1 1
    double *d_kinv = nullptr;
    double *d_u = nullptr;
    double *d_invs = nullptr;           // [S] 1 / (1^T K^-1 1)
};

// Coarse level of the two-level preconditioner (coarse.cu): three induced-dipole
// vectors per rigid body, the inverse of their model operator, and what the A-DEF1
// correction reads every iteration.  Buffers only grow; `gen` is the geometry generation
// they describe.
struct CoarseSpace {
    long long gen = -1;
    bool active = false, failed = false;
    int nbc = 0, nc = 0, np = 0;        // coarse bodies, unknowns (3 nbc), padded order
    int nmodes = 0, K2 = 0;             // half-space wave vectors, padded 2*nmodes
    long long npairs = 0;               // ordered near body pairs
    double kc = 0.0;                    // wave-vector cut used
    int *cidx = nullptr;                // [B] coarse index of a body or -1
    int *cbody = nullptr;               // [nbc] body of a coarse index
    double *zq = nullptr;               // [3N] the bead's values in its body's three columns
    double *zp = nullptr;               // [3B] body-potential rows of the columns
    double4 *cent = nullptr;            // [B] centroid, bounding radius in .w
    double *basis = nullptr;            // [6 (N+B)] right-hand sides and solutions of the basis
    int *phead = nullptr, *pcount = nullptr;  // [nbc] near pairs of each coarse body
    int *pair_a = nullptr, *pair_b = nullptr; // [npairs]
    long long *woff = nullptr;          // [npairs] first W value of the pair
    float *W = nullptr;                 // per pair: [n_a][3] real-space blocks M_real Z_q
    float4 *kv = nullptr;               // [nmodes] (mx, my, mz, sqrt w)
    int4 *rows = nullptr;               // [nrows] runs of consecutive mz: (mx, my, mz0, first mode)
    int nrows = 0, bs = 128;            // runs; threads per body CTA of the A~ Z y kernel
    size_t model_smem = 0;              // dynamic shared memory of the A~ Z y kernel
    int model_split = 1;                // threads per bead of the A~ Z y kernel
    // sparse level (coarse problems above max_dense unknowns): near-pair blocks, PCG
    int max_dense = 12288, pcg_iters = 0;  // above max_dense: pcg_iters CG steps (0: no coarse level)
    bool sparse = false;
    int nspmv = 0, nvec = 0;            // blocks of the PCG kernels (partial sums per block)
    double *Cblk = nullptr;             // [npairs][9] C_ab of each ordered near pair
    double *Dblk = nullptr;             // [nbc][9] inverse diagonal blocks
    double *pr = nullptr, *pz = nullptr, *pp = nullptr, *pq = nullptr;  // [nc] CG vectors
    double *part_pq = nullptr, *part_rz = nullptr;  // per-iteration block partial sums
    double *pu = nullptr;               // [K2] F^T p of the current CG step
    size_t cap_Cblk = 0, cap_Dblk = 0, cap_pr = 0, cap_pz = 0, cap_pp = 0, cap_pq = 0, cap_part_pq = 0,
           cap_part_rz = 0, cap_pu = 0;
    float *F = nullptr;                 // [nc][K2] scaled structure factors
    double *fpart = nullptr;            // [chunks][K2] partial column sums of F
    double *C = nullptr;                // [np][np] coarse operator (assembled in FP64)
    float *Ci = nullptr;                // [np][np] FP32 copy of C, inverted in place
    float *R = nullptr, *Fc = nullptr, *Dinv = nullptr;   // Gauss-Jordan panels (FP32)
    double *g = nullptr, *y = nullptr;  // [nc] restricted residual, coarse solution
    float *u = nullptr;                 // [K2] wave coefficients of Z y
    double *t = nullptr;                // [N+B] r - A~ Z y
    size_t cap_cidx = 0, cap_cbody = 0, cap_zq = 0, cap_zp = 0, cap_cent = 0, cap_basis = 0, cap_phead = 0,
           cap_pcount = 0, cap_pair_a = 0, cap_pair_b = 0, cap_woff = 0, cap_W = 0, cap_kv = 0, cap_F = 0,
           cap_fpart = 0, cap_C = 0, cap_Ci = 0, cap_R = 0, cap_Fc = 0, cap_Dinv = 0, cap_g = 0, cap_y = 0,
           cap_u = 0, cap_t = 0, cap_rows = 0;
};

// ---- lockstep batches (batchsolve.cu) ----------------------------------------------
// One replica of a lockstep batch: the addresses and constants every batched kernel reads
// for it, copied from its handle after the replica's set-up.  A batched kernel runs one
// CTA per work item (replica, local block) and calls the same per-block body as the
// single-system kernel with this replica's arguments.
enum BatchVec { BV_V = 0, BV_Z, BV_W, BV_R, BV_B, BV_X, BV_RR, BV_SIN, BV_SZ, BV_COUNT };

struct BatchRep {
    int N, B, n, vblk;               // beads, bodies, unknowns, blocks of the vector kernels
    int ntiles, nclus, m, pad0;      // mesh tiles, 32-bead clusters, restart length
    int Ng[3], ntd[3], zp32, zp64;   // mesh nodes and tiles per dimension, contraction pitches
    int coarse, nbc, nc, np;         // two-level coarse level (coarse = 1: active, dense)
    int nmodes, K2, nrows, pad1;
    long long goff, soff;            // the replica's mesh and half spectrum in the batch buffers
    double hm[3], halfL[3], inv_eta[3];
    double xiterm, prefac, coeff_phi, selfc;
    double Linv[3];
    // geometry
    const float4 *pos32;
    const double4 *pos64;
    const int4 *wstart;
    const int *tile_start, *tile_beads;
    float *q32, *phi32;
    double *q64, *phi64;
    // real space (stored values)
    const long long *head, *voff;
    const int *count, *pair_j, *members, *slots;
    const unsigned *masks;
    const float *vals32;
    const double *vals64;
    float *acc32;
    double *acc64;
    const uint32_t *body;
    // bodies and preconditioners
    const int *body_start, *body_members, *bsize;
    const uint8_t *rigid;
    const int *body_shape, *shape_n, *shape_vec;
    const long long *shape_mat;
    const double *kinv, *uvec, *inv_s;
    const int *cbody, *cidx, *phead, *pcount, *pair_b;
    const long long *woff;
    const double *zq, *zpv;
    const float *W, *Ci, *F;
    const float4 *kv;
    const int4 *rows;
    double *cg, *cy, *fpart, *ct;
    float *cu;
    // Krylov workspace of the replica's handle
    double *vec[BV_COUNT];
    double *partial, *hcol, *yvec, *H, *cs, *sn, *g;
};

// The precision-dependent arrays of a batch replica.
template <typename R> __device__ __forceinline__ const typename Prec<R>::R4 *brep_pos(const BatchRep &b) {
    if constexpr (sizeof(R) == 4) return b.pos32;
    else return b.pos64;
}
template <typename R> __device__ __forceinline__ R *brep_q(const BatchRep &b) {
    if constexpr (sizeof(R) == 4) return b.q32;
    else return b.q64;
}
template <typename R> __device__ __forceinline__ R *brep_phi(const BatchRep &b) {
    if constexpr (sizeof(R) == 4) return b.phi32;
    else return b.phi64;
}
template <typename R> __device__ __forceinline__ const R *brep_vals(const BatchRep &b) {
    if constexpr (sizeof(R) == 4) return b.vals32;
    else return b.vals64;
}
template <typename R> __device__ __forceinline__ R *brep_acc(const BatchRep &b) {
    if constexpr (sizeof(R) == 4) return b.acc32;
    else return b.acc64;
}

// Work lists of the batched kernels: item k = (replica, local block) of CTA k.
enum BatchList {
    BL_TILES = 0,   // mesh tiles
    BL_CLUSTERS,    // 32-bead clusters
    BL_CLELEMS,     // cluster slots, 256 per block
    BL_VEC,         // vector blocks (vblk per replica, grid-stride over the replica's rows)
    BL_BODYWARPS,   // bodies, 8 per block (one warp each)
    BL_BODIES,      // bodies, one per block
    BL_CBODIES,     // coarse bodies, one per block
    BL_GEMV,        // coarse rows, 8 per block (one warp each)
    BL_FCHUNK,      // 8-row chunks of the structure factors
    BL_FCOL,        // structure-factor columns, 8 per block (one warp each)
    BL_COUNT
};

// Replicas of one mesh size: consecutive in the batch mesh buffers, transformed by one
// batched cuFFT plan per direction and precision ([0] FP64, [1] FP32).
struct BatchFftGroup {
    int grid[3] = {0, 0, 0};
    long long goff = 0, soff = 0;
    std::vector<int> reps;
    cufftHandle fwd[2] = {0, 0}, inv[2] = {0, 0};
};

// Kernel classes timed by the built-in profiler (CUDA events on the handle's stream).
enum ProfId {
    PROF_SPREAD = 0,
    PROF_FFT,
    PROF_SCALE,
    PROF_CONTRACT,
    PROF_REAL,
    PROF_CONTRACT_FORCE,
    PROF_REAL_FORCE,
    PROF_KRYLOV,
    PROF_BODY,
    PROF_GEOMETRY,
    PROF_PRECOND,
    PROF_COARSE,
    PROF_COUNT
};

struct Profiler {
    bool on = false;
    std::vector<cudaEvent_t> pool;                 // reusable events
    size_t used = 0;
    std::vector<std::pair<int, size_t>> marks;     // (class, index of the start event)
};

}  // namespace cr

// A lockstep batch over existing handles (batchsolve.cu).
struct cr_batch {
    int n = 0;
    std::vector<cr_handle *> handles;
    std::string last_error;
    int support = 0, m = 0, precision = 0, precond = 0;
    cudaStream_t stream = nullptr, side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev0 = nullptr, ev1 = nullptr;
    // per-replica descriptors
    std::vector<cr::BatchRep> reps;
    cr::BatchRep *d_reps = nullptr;
    // work lists: the lists the launchers read (d_items, n_items) point into one of two
    // device slots, [0] every live replica, [1] the replicas of the current Arnoldi step
    int2 *d_items[cr::BL_COUNT] = {};
    int n_items[cr::BL_COUNT] = {};
    int2 *slot_base[2] = {nullptr, nullptr};
    size_t slot_cap[2] = {0, 0};
    int2 *slot_items[2][cr::BL_COUNT] = {};
    int slot_n[2][cr::BL_COUNT] = {};
    int2 *pin_items[2] = {nullptr, nullptr};       // pinned staging of each slot's upload
    size_t pin_cap[2] = {0, 0};
    std::vector<int2> h_full[cr::BL_COUNT];        // items of the live replicas, replica after replica
    std::vector<long long> rep_range[cr::BL_COUNT];  // [2 n] first and end item of each replica
    std::vector<int> step_set;                     // replicas of the lists in slot 1
    // stage masks: [0] Arnoldi step, [1] cycle end, [2] cycle start, [3] all
    int *d_mask = nullptr;
    int *h_mask = nullptr;           // pinned [4 n]
    // batch mesh buffers (every replica's mesh and half spectrum, grouped by size)
    long long G = 0, S = 0;
    float *grid32 = nullptr, *scale32 = nullptr;
    double *grid64 = nullptr, *scale64 = nullptr;
    cufftComplex *spec32 = nullptr;
    cufftDoubleComplex *spec64 = nullptr;
    std::vector<cr::BatchFftGroup> groups;
    std::vector<int> rep_group;      // group of each replica
    int contract_threads = 256;
    size_t contract_smem32 = 0, contract_smem64 = 0;
    int cond_threads = 64;
    size_t cond_smem = 0;
    int model_threads = 128, model_split = 1;
    size_t model_smem = 0;
    // solver state (device, contiguous over replicas) and its pinned mirrors
    void *d_state = nullptr, *h_state = nullptr;  // [n] Arnoldi states
    double *d_norm2 = nullptr, *h_norm2 = nullptr; // [2 n] squared norms
    double *d_scal = nullptr, *h_scal = nullptr;   // [2 n] per-replica scalars of a stage
    long long launches = 0, fft_execs = 0, steps = 0;
    double phase_ms[3] = {0, 0, 0};  // last solve: first join (host), rounds (device), whole call (host)
    std::vector<double> h_grid_check;  // derived grid and box of each replica at creation
};

struct cr_handle {
    cr_params user{};
    cr_derived d{};
    double L[3] = {0, 0, 0};
    double field[3] = {0, 0, 0};
    int N = 0, B = 0;
    bool have_topology = false;
    cudaStream_t stream = nullptr;
    std::string last_error;

    // topology
    uint32_t *d_body = nullptr;       // [N]
    uint8_t *d_rigid = nullptr;       // [B]
    double *d_Q = nullptr;            // [B]
    int *d_bsize = nullptr;           // [B]
    int *d_body_start = nullptr;      // [B+1] CSR of members
    int *d_body_members = nullptr;    // [N]
    double4 *d_bpos = nullptr;        // [B] body centres
    std::vector<int> h_body_start, h_body_members;  // host copy of the member lists
    cr::ConductorPrecond cond;
    cr::CoarseSpace coarse;

    // tables on the host (FP64)
    std::vector<double> h_phiq, h_gradphiq;

    // mesh tiling
    int tile = 8;                     // tile edge in nodes
    int spread_mode = 0;              // 0: register columns where compiled (T = 8, P = 9/11); 1: shared atomics
    int ntiles_dim[3] = {0, 0, 0};
    int ntiles = 0;

    cr::MeshBuffers<double> m64;
    cr::MeshBuffers<float> m32;
    cr::Geometry geo;
    cr::RealSpace rs;
    cr::Krylov kry;
    cr::Correction corr;

    // scratch
    double *d_tmp_n = nullptr;        // [N+B]
    double *d_tmp_n2 = nullptr;       // [N+B]
    double *d_force = nullptr;        // [3N]
    int *d_flag = nullptr;            // device error flag
    void *d_sort_tmp = nullptr;       // CUB temporary storage
    size_t sort_tmp_bytes = 0;
    int *d_keys = nullptr, *d_keys_alt = nullptr, *d_vals = nullptr, *d_vals_alt = nullptr;  // [N]
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cr::Profiler prof;
    long long launches = 0;           // kernels of this library launched (all entry points)
    long long fft_execs = 0;          // cuFFT executions
    // staging for cr_compute_host
    double *d_io_pos = nullptr, *d_io_bpos = nullptr, *d_io_q = nullptr, *d_io_phi = nullptr, *d_io_force = nullptr;
    // rigid-body stepper: body force and torque, per-body move sizes
    double *d_bf = nullptr, *d_bt = nullptr, *d_moves = nullptr;
    // solver graphs: capture one Arnoldi step per geometry when a stream is set
    int use_graphs = 1;
    // real-space kernel values: CR_REALSPACE_* flags, evaluated on the fly instead of stored
    int rs_onfly = 0;
    int n_sm = 0;                     // multiprocessors of the device
    // the wave-space part of an operator application runs on `side` (highest stream
    // priority) while the real-space product runs on `stream`
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    long long geo_gen = 0;
    long long graph_launches = 0;
    // learned guess: caller directions for the next solve [CR_MAX_GUESS_DIRECTIONS][N+B]
    double *d_guess = nullptr;
    int n_guess = 0;
};

namespace cr {

// Error plumbing: record the message on the handle and return a status.
int fail(cr_handle *h, int status, const std::string &msg);
int check_cuda(cr_handle *h, cudaError_t e, const char *what);
int check_cufft(cr_handle *h, cufftResult r, const char *what);

#define CR_TRY(expr)                      \
    do {                                  \
        int _st = (expr);                 \
        if (_st != CR_OK) return _st;     \
    } while (0)
#define CR_CUDA(h, expr) CR_TRY(::cr::check_cuda((h), (expr), #expr))
#define CR_CUFFT(h, expr) CR_TRY(::cr::check_cufft((h), (expr), #expr))
#define CR_LAUNCH(h, what)                                                 \
    do {                                                                   \
        ++(h)->launches;                                                   \
        CR_TRY(::cr::check_cuda((h), cudaGetLastError(), (what)));         \
    } while (0)

// Profiler marks: prof_begin returns a token passed to prof_end (no-ops when off).
long prof_begin(cr_handle *h, int id);
void prof_end(cr_handle *h, long token);
struct ProfScope {
    cr_handle *h;
    long tok;
    ProfScope(cr_handle *h_, int id) : h(h_), tok(prof_begin(h_, id)) {}
    ~ProfScope() { prof_end(h, tok); }
};

template <typename T> int dalloc(cr_handle *h, T **p, size_t count) {
    if (*p) { cudaFree(*p); *p = nullptr; }
    if (count == 0) return CR_OK;
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(h, e == cudaErrorMemoryAllocation ? CR_OUT_OF_MEMORY : CR_CUDA_ERROR,
                    std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return CR_OK;
}
template <typename T> void dfree(T **p) {
    if (*p) cudaFree(*p);
    *p = nullptr;
}

inline int grid_size(const cr_handle *h) { return h->d.grid[0] * h->d.grid[1] * h->d.grid[2]; }
inline int spec_size(const cr_handle *h) { return h->d.grid[0] * h->d.grid[1] * (h->d.grid[2] / 2 + 1); }
inline int blocks_for(long n, int threads) { return (int)((n + threads - 1) / threads); }

// ---- module entry points (mesh.cu, realspace.cu, body.cu, solver.cu) ----
template <typename R> int mesh_init(cr_handle *h, MeshBuffers<R> &m);
template <typename R> void mesh_free(MeshBuffers<R> &m);
int geometry_alloc(cr_handle *h);
void geometry_free(cr_handle *h);
// Positions (device, double[N*3]) -> wrapped positions, window starts, tile bins,
// neighbour list within rc.
int geometry_update(cr_handle *h, const double *d_pos, const double *d_body_pos);
// Charges (double) -> precision copy used by the operator kernels.
template <typename R> int cast_charges(cr_handle *h, MeshBuffers<R> &m, const double *d_q);
// out[i] = (double) in[i]
template <typename R> int cast_to_double(cr_handle *h, const R *in, double *out, long n);
// Wave-space potential into m.phi (R) for the charges in m.q.
template <typename R> int wave_potential(cr_handle *h, MeshBuffers<R> &m);
// Wave-space force into m.force (R) for the charges in m.q.
template <typename R> int wave_force(cr_handle *h, MeshBuffers<R> &m);
// Spread m.q into m.grid only.
template <typename R> int spread_only(cr_handle *h, MeshBuffers<R> &m);
// Real-space: out_i = Phi_b(i) - (phi_k + self q + sum T q)   (phi_body != NULL)
//             out_i = phi_k + self q + sum T q               (phi_body == NULL)
//             out_i = sum T q only (rows_only; real_space_rows then adds the rest)
template <typename R>
int real_space_apply(cr_handle *h, MeshBuffers<R> &m, const double *phi_body, double *out, bool rows_only = false);
template <typename R> int real_space_rows(cr_handle *h, MeshBuffers<R> &m, const double *phi_body, double *out);
// Forces: out = wave force (m.force) + q E0 + real-space force for FP64 charges q64.
template <typename R> int real_space_force(cr_handle *h, MeshBuffers<R> &m, const double *q64, double *force_out);
int realspace_alloc(cr_handle *h);
void realspace_free(cr_handle *h);
// Clusters and cluster pairs of the current positions.
int realspace_build(cr_handle *h);
// Virial tensors (xx, xy, xz, yy, yz, zz) of the FP64 charges q64 at the current geometry:
// real-space part into out[0..5]; wave-space part of the charges in m64.q into out[0..5]
// and the wave energy into out[6].
int real_space_virial(cr_handle *h, const double *q64, double *out);
int wave_virial(cr_handle *h, double *out);
int realspace_prepare(cr_handle *h, int precision);
// CR_TIMEOUT (and the error word cleared) when a bounded wait of the streamed product ran
// out since the last check; synchronises the stream.
int realspace_check(cr_handle *h);
int mesh_set_tile(cr_handle *h, int T);
int neighbor_list_build(cr_handle *h, double r_list, int *d_count, int64_t *d_head, int *d_list,
                        int64_t capacity, int64_t *total);
// Body rows y[N+b] = sum_{i in b} x_i (FP64).
int body_sums(cr_handle *h, const double *x, double *y);
// Member lists of the bodies from d_body (stable device sort).
int topology_build(cr_handle *h);
int objective(cr_handle *h, double *rhs);
// The handle's preconditioner (diagonal or conductor response).
int precondition(cr_handle *h, const double *x, double *y);
int conductor_setup(cr_handle *h);
int conductor_apply(cr_handle *h, const double *x, double *y);
void conductor_free(cr_handle *h);
// Coarse level of CR_PRECOND_TWO_LEVEL for the current geometry (no-op otherwise or when
// already built); coarse_apply is the whole two-level preconditioner.
int coarse_prepare(cr_handle *h);
int coarse_apply(cr_handle *h, const double *x, double *z);
void coarse_free(cr_handle *h);
// y = A x in the given precision (full operator).
int apply_operator(cr_handle *h, const double *x, double *y, int precision);
// Solve A x = b (x holds the warm start).
int solve(cr_handle *h, double *x, const double *b, cr_solve_stats *st);
// learned correction of the preconditioner (correction.cu)
int correction_prepare(cr_handle *h);
void correction_free(cr_handle *h);
int correction_add(cr_handle *h, const double *v, double *z);
int precondition_step(cr_handle *h, const double *v, double *z);
int correction_decide(cr_handle *h, int precision, const double *r, double *w);
int correction_samples(cr_handle *h, int max_dirs, uint16_t *d_x, float *d_t, int *rows);
// out[0..k) = V[0..k)^T w over the N + B unknowns (device result)
int dots(cr_handle *h, int k, const double *V, const double *w, double *out);
int body_force_torque(cr_handle *h, const double *pos, const double *bpos, const double *force, double *bf,
                      double *bt);
int brownian_step(cr_handle *h, const cr_brownian_params *bp, long long step, const double *radius,
                  const double *force, double *pos, double *bpos);
int krylov_alloc(cr_handle *h);
void krylov_free(cr_handle *h);

// ---- lockstep batch stages: one launch per stage over the replicas whose entry in the
// mask (device, [n]) is nonzero; xin / yout select vectors of the Krylov workspace ----
int batch_fail(cr_batch *bt, int status, const std::string &msg);
int batch_check(cr_batch *bt, cudaError_t e, const char *what);
// charges of the input vector into the operator precision (mesh.cu)
template <typename R> int batch_cast(cr_batch *bt, const int *mask, int xin, cudaStream_t s);
// wave-space potential: spread, transforms by size group, influence function, contract
// (mesh.cu); group_live[g] = 0 skips a size group whose replicas are all masked out
template <typename R> int batch_wave(cr_batch *bt, const int *mask, const std::vector<char> &group_live, cudaStream_t s);
// real-space sums into the rows of yout (realspace.cu), then the full rows
template <typename R> int batch_real(cr_batch *bt, const int *mask, int yout, cudaStream_t s);
template <typename R> int batch_rows(cr_batch *bt, const int *mask, int xin, int yout, cudaStream_t s);
// body rows yout[N + b] = sum of xin over body b (body.cu)
int batch_body_sums(cr_batch *bt, const int *mask, int xin, int yout, cudaStream_t s);
// the batch's preconditioner zout = P xin (body.cu, conductor.cu, coarse.cu)
int batch_diag(cr_batch *bt, const int *mask, int xin, int zout, cudaStream_t s);
int batch_conductor(cr_batch *bt, const int *mask, int xin, bool from_coarse, int zout, cudaStream_t s);
int batch_coarse(cr_batch *bt, const int *mask, int xin, int zout, cudaStream_t s);
// dynamic shared memory of the batched kernels (process-wide attributes, only grown)
int batch_mesh_attrs(cr_batch *bt);
int batch_coarse_attrs(cr_batch *bt);

}  // namespace cr
