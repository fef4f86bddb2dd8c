// batchsolve.cu -- many independent systems solved in lockstep, one launch per stage.
//
// cr_batch_compute (batch.cu) runs the single-system solver of each replica on its own
// stream; every replica then pays its own ~25 launches per Arnoldi iteration, and small
// replicas leave the GPU waiting on launches.  A lockstep batch instead advances every
// unconverged replica by one Arnoldi step per round, and each stage of that step is ONE
// launch over all replicas: a work list of (replica, local block) items, the replica's
// addresses taken from a device table of descriptors (BatchRep) and the per-block body
// shared with the single-system kernel.  The stages of a step (FP32 operator, CR_MIXED):
//
//   gather V_j | preconditioner (restrict, coarse GEMV, F^T y, model, conductor response,
//   prolong) | scatter Z_j | cast charges | spread | R2C per mesh-size group | influence
//   function | C2R per group | contract  (beside: cluster gather, stored-value product) |
//   rows | body sums | two Gram-Schmidt passes (dots, reduction, projection) | norm |
//   Hessenberg column and Givens rotation (one thread per replica) | V_{j+1} | advance
//
// Replicas of one mesh size sit consecutively in the batch's mesh buffers and are
// transformed by one batched cuFFT plan, so the transforms take one launch per size, not
// per replica.  The per-replica solver logic is that of the single-system solver
// (solver.cu): flexible GMRES with FP64 Arnoldi, in CR_MIXED FP32 cycles inside FP64
// iterative refinement (three decades per cycle while the target is more than four
// decades away, then to 0.3 of it), the cycle's least-squares update solved on the
// device, the refinement residual b - A64 x from the batched FP64 operator.  A replica
// whose cycle ends leaves the Arnoldi mask for one round (update, FP64 residual, norm)
// and re-enters with its next cycle; converged replicas drop out of every mask.
//
// Work that runs once per solve stays per replica, as tasks of a pool of host threads
// with one stream each: the geometry (tiles, clusters, masks, stored values), the
// right-hand side, the coarse level of the two-level preconditioner, and the FP64 force
// pass after the solve.  A replica joins the rounds as soon as its set-up is done and
// leaves for its force pass as soon as it has converged, so the three overlap on the GPU;
// the task streams take the highest priority (a set-up is a latency-bound chain of small
// kernels) and the rounds the lowest.  Each round's work lists hold only the replicas
// taking part in it.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "cr_internal.cuh"

namespace cr {

int batch_fail(cr_batch *bt, int status, const std::string &msg) {
    bt->last_error = msg;
    return status;
}

int batch_check(cr_batch *bt, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return CR_OK;
    cudaGetLastError();
    return batch_fail(bt, e == cudaErrorMemoryAllocation ? CR_OUT_OF_MEMORY : CR_CUDA_ERROR,
                      std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

constexpr int kThreads = 256;

// Arnoldi state of one replica (the single solver's captured-step state).
struct BState {
    int j;          // columns completed in this cycle
    int stop;       // 1: tolerance met or breakdown; 2: non-finite norm
    int frozen;     // set once a stopping column is counted
    int pad;
    double res;     // |g[j]| after the last counted column
    double inv_hn;  // 1 / ||w|| of the column being added
    double atol;    // absolute tolerance of this cycle
};

#define BATCH_ITEM()                        \
    const int2 it = items[blockIdx.x];      \
    if (!mask[it.x]) return;                \
    const BatchRep &r = reps[it.x]

// sin = V_j
__global__ void gather_v_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                const int *__restrict__ mask, const BState *__restrict__ st) {
    BATCH_ITEM();
    const size_t off = (size_t)st[it.x].j * r.n;
    const double *V = r.vec[BV_V];
    double *dst = r.vec[BV_SIN];
    for (int i = it.y * blockDim.x + threadIdx.x; i < r.n; i += r.vblk * blockDim.x) dst[i] = V[off + i];
}

// Z_j = sz
__global__ void scatter_z_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                 const int *__restrict__ mask, const BState *__restrict__ st) {
    BATCH_ITEM();
    const int j = st[it.x].j;
    if (j >= r.m) return;
    const double *src = r.vec[BV_SZ];
    double *Z = r.vec[BV_Z] + (size_t)j * r.n;
    for (int i = it.y * blockDim.x + threadIdx.x; i < r.n; i += r.vblk * blockDim.x) Z[i] = src[i];
}

// partial[blk * kmax + c] = sum over this block's rows of a_c[i] * w[i]   (c < k), with
// a_c = A + c n; k = min(j + 1, kmax) from the state when use_state, else kmax.  Eight
// vectors per pass, the block's warps reduced in a fixed order.
constexpr int kDotChunk = 8;
__global__ void __launch_bounds__(kThreads) dots_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                                        const int *__restrict__ mask, const BState *__restrict__ st,
                                                        int use_state, int kmax, int va, int vw) {
    __shared__ double red[kThreads / 32][kDotChunk];
    BATCH_ITEM();
    const int k = use_state ? min(st[it.x].j + 1, kmax) : kmax;
    const int n = r.n, blk = it.y, nblk = r.vblk;
    const double *A = r.vec[va], *w = r.vec[vw];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j0 = 0; j0 < k; j0 += kDotChunk) {
        double acc[kDotChunk];
#pragma unroll
        for (int c = 0; c < kDotChunk; ++c) acc[c] = 0.0;
        const int kc = min(kDotChunk, k - j0);
        for (int i = blk * blockDim.x + threadIdx.x; i < n; i += nblk * blockDim.x) {
            const double wi = w[i];
#pragma unroll
            for (int c = 0; c < kDotChunk; ++c)
                if (c < kc) acc[c] += A[(size_t)(j0 + c) * n + i] * wi;
        }
#pragma unroll
        for (int c = 0; c < kDotChunk; ++c) {
            for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
            if (lane == 0) red[warp][c] = acc[c];
        }
        __syncthreads();
        if (threadIdx.x < kc) {
            double t = 0.0;
            for (int q = 0; q < kThreads / 32; ++q) t += red[q][threadIdx.x];
            r.partial[(size_t)blk * kmax + j0 + threadIdx.x] = t;
        }
        __syncthreads();
    }
}

// Block sums of dots_kernel, one warp per (replica, c), in block order.  out_norm: the
// single sum goes to norm2[replica]; else to hcol[out_off + c].
__global__ void reduce_kernel(const BatchRep *__restrict__ reps, int n_reps, const int *__restrict__ mask,
                              const BState *__restrict__ st, int use_state, int kmax, int out_norm, int out_off,
                              double *__restrict__ norm2) {
    const int rep = blockIdx.x / kmax, c = blockIdx.x - rep * kmax;
    if (rep >= n_reps || !mask[rep]) return;
    const BatchRep &r = reps[rep];
    const int k = use_state ? min(st[rep].j + 1, kmax) : kmax;
    if (c >= k) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < r.vblk; b += 32) s += r.partial[(size_t)b * kmax + c];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) {
        if (out_norm) norm2[rep] = s;
        else r.hcol[out_off + c] = s;
    }
}

// w -= sum_c hv[c] V_c,  hv = hcol + pass (m + 1), c < min(j + 1, m + 1)
__global__ void project_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                               const int *__restrict__ mask, const BState *__restrict__ st, int pass) {
    BATCH_ITEM();
    const int k = min(st[it.x].j + 1, r.m + 1);
    const double *V = r.vec[BV_V], *hv = r.hcol + (size_t)pass * (r.m + 1);
    double *w = r.vec[BV_W];
    for (int i = it.y * blockDim.x + threadIdx.x; i < r.n; i += r.vblk * blockDim.x) {
        double s = w[i];
#pragma unroll 8
        for (int c = 0; c < k; ++c) s -= hv[c] * V[(size_t)c * r.n + i];
        w[i] = s;
    }
}

// Hessenberg column j with its Givens rotations and the stopping test (one thread per
// replica; the single solver's arnoldi_column_kernel).
__global__ void column_kernel(const BatchRep *__restrict__ reps, int n_reps, const int *__restrict__ mask,
                              BState *__restrict__ st) {
    const int rep = blockIdx.x * blockDim.x + threadIdx.x;
    if (rep >= n_reps || !mask[rep]) return;
    const BatchRep &r = reps[rep];
    BState &s = st[rep];
    s.inv_hn = 0.0;
    if (s.frozen) return;
    const int j = s.j, m = r.m;
    if (j >= m) return;
    const double *hcol = r.hcol;
    double *H = r.H, *cs = r.cs, *sn = r.sn, *g = r.g;
    const double *h1 = hcol, *h2 = hcol + (m + 1);
    const double hn = sqrt(fmax(0.0, hcol[2 * (m + 1)]));
    if (!isfinite(hn)) {
        s.stop = 2;
        return;
    }
    for (int k = 0; k <= j; ++k) H[(size_t)k * m + j] = h1[k] + h2[k];
    H[(size_t)(j + 1) * m + j] = hn;
    for (int k = 0; k < j; ++k) {
        const double a = H[(size_t)k * m + j], c = H[(size_t)(k + 1) * m + j];
        H[(size_t)k * m + j] = cs[k] * a + sn[k] * c;
        H[(size_t)(k + 1) * m + j] = -sn[k] * a + cs[k] * c;
    }
    const double a = H[(size_t)j * m + j], c = H[(size_t)(j + 1) * m + j];
    const double den = hypot(a, c);
    cs[j] = den > 0 ? a / den : 1.0;
    sn[j] = den > 0 ? c / den : 0.0;
    H[(size_t)j * m + j] = den;
    H[(size_t)(j + 1) * m + j] = 0.0;
    g[j + 1] = -sn[j] * g[j];
    g[j] = cs[j] * g[j];
    s.res = fabs(g[j + 1]);
    s.inv_hn = hn > 0 ? 1.0 / hn : 0.0;
    if (fabs(g[j + 1]) <= s.atol || hn == 0.0) s.stop = 1;
}

// V_{j+1} = w / ||w||
__global__ void next_v_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                              const int *__restrict__ mask, const BState *__restrict__ st) {
    BATCH_ITEM();
    const BState s = st[it.x];
    if (s.frozen || s.j >= r.m || s.inv_hn == 0.0) return;
    const double *w = r.vec[BV_W];
    double *V = r.vec[BV_V] + (size_t)(s.j + 1) * r.n;
    for (int i = it.y * blockDim.x + threadIdx.x; i < r.n; i += r.vblk * blockDim.x) V[i] = s.inv_hn * w[i];
}

__global__ void advance_kernel(const BatchRep *__restrict__ reps, int n_reps, const int *__restrict__ mask,
                               BState *__restrict__ st) {
    const int rep = blockIdx.x * blockDim.x + threadIdx.x;
    if (rep >= n_reps || !mask[rep]) return;
    BState &s = st[rep];
    if (s.frozen) return;
    if (s.stop == 2) {
        s.frozen = 1;
        return;
    }
    s.j += 1;
    if (s.stop || s.j >= reps[rep].m) s.frozen = 1;
}

// End of a cycle: y = H^-1 g over the j completed columns (upper triangular, rotated),
// one thread per replica.
__global__ void cycle_solve_kernel(const BatchRep *__restrict__ reps, int n_reps, const int *__restrict__ mask,
                                   const BState *__restrict__ st) {
    const int rep = blockIdx.x * blockDim.x + threadIdx.x;
    if (rep >= n_reps || !mask[rep]) return;
    const BatchRep &r = reps[rep];
    const int j = st[rep].j, m = r.m;
    const double *H = r.H, *g = r.g;
    double *y = r.yvec;
    for (int rr = j - 1; rr >= 0; --rr) {
        double acc = g[rr];
        for (int k = rr + 1; k < j; ++k) acc -= H[(size_t)rr * m + k] * y[k];
        y[rr] = H[(size_t)rr * m + rr] != 0.0 ? acc / H[(size_t)rr * m + rr] : 0.0;
    }
}

// x += sum_c y_c Z_c over the cycle's columns; from_zero: the correction is summed from
// zero first and then added (the refinement step x += d with d = Z y), else in place.
__global__ void update_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                              const int *__restrict__ mask, const BState *__restrict__ st, int from_zero) {
    BATCH_ITEM();
    const int j = st[it.x].j;
    const double *Z = r.vec[BV_Z], *y = r.yvec;
    double *x = r.vec[BV_X];
    for (int i = it.y * blockDim.x + threadIdx.x; i < r.n; i += r.vblk * blockDim.x) {
        if (from_zero) {
            double s = 0.0;
            for (int c = 0; c < j; ++c) s += y[c] * Z[(size_t)c * r.n + i];
            x[i] += s;
        } else {
            double s = x[i];
            for (int c = 0; c < j; ++c) s += y[c] * Z[(size_t)c * r.n + i];
            x[i] = s;
        }
    }
}

// out = b - out
__global__ void residual_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                const int *__restrict__ mask, int out) {
    BATCH_ITEM();
    const double *b = r.vec[BV_B];
    double *y = r.vec[out];
    for (int i = it.y * blockDim.x + threadIdx.x; i < r.n; i += r.vblk * blockDim.x) y[i] = b[i] - y[i];
}

__global__ void copy_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                            const int *__restrict__ mask, int src, int dst) {
    BATCH_ITEM();
    const double *a = r.vec[src];
    double *b = r.vec[dst];
    for (int i = it.y * blockDim.x + threadIdx.x; i < r.n; i += r.vblk * blockDim.x) b[i] = a[i];
}

// Start of a cycle: V_0 = scal[rep] * src (scal = 1 / beta).
__global__ void start_v_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                               const int *__restrict__ mask, const double *__restrict__ scal, int src) {
    BATCH_ITEM();
    const double a = scal[it.x];
    const double *x = r.vec[src];
    double *V = r.vec[BV_V];
    for (int i = it.y * blockDim.x + threadIdx.x; i < r.n; i += r.vblk * blockDim.x) V[i] = a * x[i];
}

// Cycle state and g = (beta, 0, ...): scal[n + rep] = beta, scal[2 n + rep] = the cycle's
// absolute tolerance.
__global__ void start_state_kernel(const BatchRep *__restrict__ reps, int n_reps, const int *__restrict__ mask,
                                   const double *__restrict__ scal, BState *__restrict__ st) {
    const int rep = blockIdx.x * blockDim.x + threadIdx.x;
    if (rep >= n_reps || !mask[rep]) return;
    const BatchRep &r = reps[rep];
    const double beta = scal[n_reps + rep];
    for (int i = 0; i <= r.m; ++i) r.g[i] = i == 0 ? beta : 0.0;
    BState s;
    s.j = 0;
    s.stop = 0;
    s.frozen = 0;
    s.pad = 0;
    s.res = beta;
    s.inv_hn = 0.0;
    s.atol = scal[2 * n_reps + rep];
    st[rep] = s;
}

int blocks_of_reps(int n) { return (n + 127) / 128; }

// ---- host side ----

enum Phase { kIdle = 0, kStart, kArnoldi, kEnd, kDone };

struct Run {
    int phase = kIdle;
    int status = CR_OK;
    double tol = 0, bnorm = 0, atol = 0, rnorm = 0;
    int maxit = 0;
    bool force_queued = false;
    int outer = 0;
    cr_solve_stats s{};
};

// Upload the work lists of the replicas in `set` (their ranges of h_full) into device slot
// `slot` (the buffer only grows, by half again, so that a growing batch reallocates rarely).
int upload_slot(cr_batch *bt, int slot, const std::vector<int> &set) {
    size_t total = 0;
    for (int k = 0; k < BL_COUNT; ++k)
        for (int i : set) total += (size_t)(bt->rep_range[k][2 * i + 1] - bt->rep_range[k][2 * i]);
    // pinned staging (one buffer per slot: the next upload into a slot comes after the
    // stream synchronisation that ends the phase reading it)
    if (total > bt->pin_cap[slot]) {
        if (bt->pin_items[slot]) cudaFreeHost(bt->pin_items[slot]);
        bt->pin_items[slot] = nullptr;
        bt->pin_cap[slot] = 0;
        const size_t cap = std::max<size_t>(total + total / 2, 1024);
        CR_TRY(batch_check(bt, cudaMallocHost((void **)&bt->pin_items[slot], cap * sizeof(int2)), "work lists"));
        bt->pin_cap[slot] = cap;
    }
    int2 *h = bt->pin_items[slot];
    size_t off[BL_COUNT], pos = 0;
    for (int k = 0; k < BL_COUNT; ++k) {
        off[k] = pos;
        for (int i : set) {
            const long long b = bt->rep_range[k][2 * i], e = bt->rep_range[k][2 * i + 1];
            if (e > b) std::memcpy(h + pos, bt->h_full[k].data() + b, (size_t)(e - b) * sizeof(int2));
            pos += (size_t)(e - b);
        }
        bt->slot_n[slot][k] = (int)(pos - off[k]);
    }
    if (total > bt->slot_cap[slot]) {
        if (bt->slot_base[slot]) cudaFree(bt->slot_base[slot]);
        bt->slot_base[slot] = nullptr;
        bt->slot_cap[slot] = 0;
        const size_t cap = std::max<size_t>(total + total / 2, 1024);
        CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->slot_base[slot], cap * sizeof(int2)), "work lists"));
        bt->slot_cap[slot] = cap;
    }
    for (int k = 0; k < BL_COUNT; ++k) bt->slot_items[slot][k] = bt->slot_base[slot] + off[k];
    if (total)
        CR_TRY(batch_check(bt, cudaMemcpyAsync(bt->slot_base[slot], h, total * sizeof(int2), cudaMemcpyHostToDevice,
                                               bt->stream),
                           "work lists upload"));
    return CR_OK;
}

// The lists the launchers read: slot 0 (the replicas of a join or of cycle ends) or slot 1
// (the replicas of the current Arnoldi step).
void use_slot(cr_batch *bt, int slot) {
    for (int k = 0; k < BL_COUNT; ++k) {
        bt->d_items[k] = bt->slot_items[slot][k];
        bt->n_items[k] = bt->slot_n[slot][k];
    }
}

// Launch shapes shared by the replicas (reset at the start of every solve).
struct Shapes {
    int model_bs = -1, model_split = -1;
};

// Descriptor of replica i after its set-up; the launch shapes grow to cover it.
int describe_rep(cr_batch *bt, int i, Shapes &sh) {
    {
        cr_handle *h = bt->handles[i];
        BatchRep &r = bt->reps[i];
        std::memset(&r, 0, sizeof(BatchRep));
        const Krylov &K = h->kry;
        r.N = h->N;
        r.B = h->B;
        r.n = K.n;
        r.vblk = K.nblocks;
        r.ntiles = h->ntiles;
        r.nclus = h->rs.nclus;
        r.m = K.m;
        for (int d = 0; d < 3; ++d) {
            r.Ng[d] = h->d.grid[d];
            r.ntd[d] = h->ntiles_dim[d];
            r.hm[d] = h->d.h[d];
            r.halfL[d] = 0.5 * h->L[d];
            r.inv_eta[d] = 1.0 / h->d.eta[d];
            r.Linv[d] = 1.0 / h->L[d];
        }
        const int P = h->d.support, Bd = 8 + P - 1;
        r.zp32 = (Bd * Bd * (P + 32) + 8 * 6 * P) * 4 <= 227 * 1024 ? P + 32 : Bd;
        r.zp64 = (Bd * Bd * (P + 32) + 8 * 6 * P) * 8 <= 227 * 1024 ? P + 32 : Bd;
        r.xiterm = h->d.xiterm;
        r.prefac = h->d.prefac;
        r.coeff_phi = h->d.quadW * h->d.prefac;
        r.selfc = h->d.selfcoeff;
        const BatchFftGroup &G = bt->groups[bt->rep_group[i]];
        size_t pos_in_group = 0;
        for (size_t q = 0; q < G.reps.size(); ++q)
            if (G.reps[q] == i) pos_in_group = q;
        const long long Gn = (long long)G.grid[0] * G.grid[1] * G.grid[2];
        const long long Sn = (long long)G.grid[0] * G.grid[1] * (G.grid[2] / 2 + 1);
        r.goff = G.goff + (long long)pos_in_group * Gn;
        r.soff = G.soff + (long long)pos_in_group * Sn;
        r.pos32 = h->m32.pos;
        r.pos64 = h->m64.pos;
        r.wstart = h->geo.wstart;
        r.tile_start = h->geo.tile_start;
        r.tile_beads = h->geo.tile_beads;
        r.q32 = h->m32.q;
        r.phi32 = h->m32.phi;
        r.q64 = h->m64.q;
        r.phi64 = h->m64.phi;
        const RealSpace &rs = h->rs;
        r.head = rs.head;
        r.voff = rs.voff;
        r.count = rs.count;
        r.pair_j = rs.pair_j;
        r.members = rs.members;
        r.slots = rs.nnz_pair;
        r.masks = rs.masks;
        r.vals32 = rs.vals32;
        r.vals64 = rs.vals64;
        r.acc32 = rs.acc32;
        r.acc64 = rs.acc64;
        r.body = h->d_body;
        r.body_start = h->d_body_start;
        r.body_members = h->d_body_members;
        r.bsize = h->d_bsize;
        r.rigid = h->d_rigid;
        const ConductorPrecond &C = h->cond;
        r.body_shape = C.d_body_shape;
        r.shape_n = C.d_shape_n;
        r.shape_vec = C.d_shape_vec;
        r.shape_mat = C.d_shape_mat;
        r.kinv = C.d_kinv;
        r.uvec = C.d_u;
        r.inv_s = C.d_invs;
        if (bt->precond != CR_PRECOND_DIAGONAL && h->B > 0) {
            bt->cond_threads = std::max(bt->cond_threads, std::min(256, std::max(64, (C.max_n + 31) / 32 * 32)));
            bt->cond_smem = std::max(bt->cond_smem, (size_t)C.max_n * sizeof(double));
        }
        const CoarseSpace &cs = h->coarse;
        if (bt->precond == CR_PRECOND_TWO_LEVEL && cs.active) {
            if (cs.sparse)
                return batch_fail(bt, CR_BAD_PARAM,
                                  "lockstep batch: a replica's coarse level uses the sparse form (too many bodies)");
            if (sh.model_bs < 0) {
                sh.model_bs = cs.bs;
                sh.model_split = cs.model_split;
            } else if (cs.bs != sh.model_bs || cs.model_split != sh.model_split) {
                return batch_fail(bt, CR_BAD_PARAM,
                                  "lockstep batch: replicas' largest bodies differ in warps (coarse model launch shape)");
            }
            bt->model_smem = std::max(bt->model_smem, cs.model_smem);
            r.coarse = 1;
            r.nbc = cs.nbc;
            r.nc = cs.nc;
            r.np = cs.np;
            r.nmodes = cs.nmodes;
            r.K2 = cs.K2;
            r.nrows = cs.nrows;
            r.cbody = cs.cbody;
            r.cidx = cs.cidx;
            r.phead = cs.phead;
            r.pcount = cs.pcount;
            r.pair_b = cs.pair_b;
            r.woff = cs.woff;
            r.zq = cs.zq;
            r.zpv = cs.zp;
            r.W = cs.W;
            r.Ci = cs.Ci;
            r.F = cs.F;
            r.kv = cs.kv;
            r.rows = cs.rows;
            r.cg = cs.g;
            r.cy = cs.y;
            r.fpart = cs.fpart;
            r.ct = cs.t;
            r.cu = cs.u;
        }
        r.vec[BV_V] = K.V;
        r.vec[BV_Z] = K.Z;
        r.vec[BV_W] = K.w;
        r.vec[BV_R] = K.r;
        r.vec[BV_B] = K.b;
        r.vec[BV_X] = K.x;
        r.vec[BV_RR] = K.rr;
        r.vec[BV_SIN] = K.sin;
        r.vec[BV_SZ] = K.sz;
        r.partial = K.partial;
        r.hcol = K.hcol;
        r.yvec = K.yvec;
        r.H = K.H;
        r.cs = K.cs;
        r.sn = K.sn;
        r.g = K.g;
    }
    bt->model_threads = sh.model_bs > 0 ? sh.model_bs * sh.model_split : 128;
    bt->model_split = sh.model_split > 0 ? sh.model_split : 1;
    return CR_OK;
}

// Work items of the replicas that just joined (kept on the host; each phase uploads the
// ranges of the replicas taking part) and the descriptor table, uploaded on the batch
// stream (between rounds: the stream is idle then).
int publish(cr_batch *bt, const std::vector<int> &joined) {
    const int n = bt->n;
    for (int k = 0; k < BL_COUNT; ++k)
        if (bt->rep_range[k].size() != 2 * (size_t)n) bt->rep_range[k].assign(2 * (size_t)n, 0);
    for (int i : joined) {
        const BatchRep &r = bt->reps[i];
        auto add = [&](int list, long long count) {
            std::vector<int2> &L = bt->h_full[list];
            bt->rep_range[list][2 * i] = (long long)L.size();
            for (long long k = 0; k < count; ++k) L.push_back(make_int2(i, (int)k));
            bt->rep_range[list][2 * i + 1] = (long long)L.size();
        };
        add(BL_TILES, r.ntiles);
        add(BL_CLUSTERS, r.nclus);
        add(BL_CLELEMS, ((long long)r.nclus * 32 + kThreads - 1) / kThreads);
        add(BL_VEC, r.vblk);
        add(BL_BODYWARPS, ((long long)r.B * 32 + kThreads - 1) / kThreads);
        add(BL_BODIES, r.B);
        add(BL_CBODIES, r.coarse ? r.nbc : 0);
        add(BL_GEMV, r.coarse ? ((long long)r.nc * 32 + kThreads - 1) / kThreads : 0);
        add(BL_FCHUNK, r.coarse && r.nmodes > 0 ? (r.nc + 7) / 8 : 0);
        add(BL_FCOL, r.coarse && r.nmodes > 0 ? ((long long)r.K2 * 32 + kThreads - 1) / kThreads : 0);
    }
    CR_TRY(batch_coarse_attrs(bt));
    return batch_check(bt,
                       cudaMemcpyAsync(bt->d_reps, bt->reps.data(), (size_t)n * sizeof(BatchRep),
                                       cudaMemcpyHostToDevice, bt->stream),
                       "descriptor upload");
}

int *mask_ptr(cr_batch *bt, int which) { return bt->d_mask + (size_t)which * bt->n; }
enum { kMaskStep = 0, kMaskEnd = 1, kMaskStart = 2, kMaskAll = 3 };

// Size groups holding at least one replica of a host mask.
std::vector<char> live_groups(cr_batch *bt, const int *hmask) {
    std::vector<char> live(bt->groups.size(), 0);
    for (int i = 0; i < bt->n; ++i)
        if (hmask[i]) live[bt->rep_group[i]] = 1;
    return live;
}

// y = A x in precision R for the replicas of mask `which`: cast, then the wave part on the
// side stream beside the real-space product, joined for the rows and body sums.
template <typename R> int batch_operator(cr_batch *bt, int which, int xin, int yout) {
    const int *mask = mask_ptr(bt, which);
    const std::vector<char> live = live_groups(bt, bt->h_mask + (size_t)which * bt->n);
    CR_TRY(batch_cast<R>(bt, mask, xin, bt->stream));
    CR_TRY(batch_check(bt, cudaEventRecord(bt->ev_fork, bt->stream), "fork"));
    CR_TRY(batch_check(bt, cudaStreamWaitEvent(bt->side, bt->ev_fork, 0), "fork"));
    const int wst = batch_wave<R>(bt, mask, live, bt->side);
    const cudaError_t je = cudaEventRecord(bt->ev_join, bt->side);
    const int rst = batch_real<R>(bt, mask, yout, bt->stream);
    CR_TRY(batch_check(bt, cudaStreamWaitEvent(bt->stream, bt->ev_join, 0), "join"));
    CR_TRY(wst);
    CR_TRY(batch_check(bt, je, "join"));
    CR_TRY(rst);
    CR_TRY(batch_rows<R>(bt, mask, xin, yout, bt->stream));
    return batch_body_sums(bt, mask, xin, yout, bt->stream);
}

int batch_operator_p(cr_batch *bt, int precision, int which, int xin, int yout) {
    return precision == CR_FP64 ? batch_operator<double>(bt, which, xin, yout)
                                : batch_operator<float>(bt, which, xin, yout);
}

int batch_precondition(cr_batch *bt, int which, int xin, int zout) {
    const int *mask = mask_ptr(bt, which);
    if (bt->precond == CR_PRECOND_TWO_LEVEL) return batch_coarse(bt, mask, xin, zout, bt->stream);
    if (bt->precond == CR_PRECOND_CONDUCTOR) return batch_conductor(bt, mask, xin, false, zout, bt->stream);
    return batch_diag(bt, mask, xin, zout, bt->stream);
}

int launch_check(cr_batch *bt, const char *what) {
    ++bt->launches;
    return batch_check(bt, cudaGetLastError(), what);
}

// Squared norms of vector v of the replicas of mask `which` into d_norm2[off + replica].
int batch_norms(cr_batch *bt, int which, int v, int off = 0) {
    const int *mask = mask_ptr(bt, which);
    BState *st = reinterpret_cast<BState *>(bt->d_state);
    if (bt->n_items[BL_VEC] == 0) return CR_OK;
    dots_kernel<<<bt->n_items[BL_VEC], kThreads, 0, bt->stream>>>(bt->d_reps, bt->d_items[BL_VEC], mask, st, 0, 1, v,
                                                                   v);
    CR_TRY(launch_check(bt, "dots_kernel"));
    reduce_kernel<<<bt->n, 32, 0, bt->stream>>>(bt->d_reps, bt->n, mask, st, 0, 1, 1, 0, bt->d_norm2 + off);
    return launch_check(bt, "reduce_kernel");
}

// One Arnoldi step of every replica in the step mask (its cycle started first where the
// start mask says so).
int batch_step(cr_batch *bt, int inner) {
    const int *mS = mask_ptr(bt, kMaskStart), *mA = mask_ptr(bt, kMaskStep);
    const int nv = bt->n_items[BL_VEC], nr = bt->n;
    const int2 *vec = bt->d_items[BL_VEC];
    BState *st = reinterpret_cast<BState *>(bt->d_state);
    cudaStream_t s = bt->stream;
    const int src = bt->precision == CR_MIXED ? BV_RR : BV_R;
    start_v_kernel<<<nv, kThreads, 0, s>>>(bt->d_reps, vec, mS, bt->d_scal, src);
    CR_TRY(launch_check(bt, "start_v_kernel"));
    start_state_kernel<<<blocks_of_reps(nr), 128, 0, s>>>(bt->d_reps, nr, mS, bt->d_scal, st);
    CR_TRY(launch_check(bt, "start_state_kernel"));
    gather_v_kernel<<<nv, kThreads, 0, s>>>(bt->d_reps, vec, mA, st);
    CR_TRY(launch_check(bt, "gather_v_kernel"));
    CR_TRY(batch_precondition(bt, kMaskStep, BV_SIN, BV_SZ));
    scatter_z_kernel<<<nv, kThreads, 0, s>>>(bt->d_reps, vec, mA, st);
    CR_TRY(launch_check(bt, "scatter_z_kernel"));
    CR_TRY(batch_operator_p(bt, inner, kMaskStep, BV_SZ, BV_W));
    const int kmax = bt->m + 1;
    for (int pass = 0; pass < 2; ++pass) {  // classical Gram-Schmidt, twice
        dots_kernel<<<nv, kThreads, 0, s>>>(bt->d_reps, vec, mA, st, 1, kmax, BV_V, BV_W);
        CR_TRY(launch_check(bt, "dots_kernel"));
        reduce_kernel<<<nr * kmax, 32, 0, s>>>(bt->d_reps, nr, mA, st, 1, kmax, 0, pass * kmax, bt->d_norm2);
        CR_TRY(launch_check(bt, "reduce_kernel"));
        project_kernel<<<nv, kThreads, 0, s>>>(bt->d_reps, vec, mA, st, pass);
        CR_TRY(launch_check(bt, "project_kernel"));
    }
    dots_kernel<<<nv, kThreads, 0, s>>>(bt->d_reps, vec, mA, st, 0, 1, BV_W, BV_W);
    CR_TRY(launch_check(bt, "dots_kernel"));
    reduce_kernel<<<nr, 32, 0, s>>>(bt->d_reps, nr, mA, st, 0, 1, 0, 2 * kmax, bt->d_norm2);
    CR_TRY(launch_check(bt, "reduce_kernel"));
    column_kernel<<<blocks_of_reps(nr), 128, 0, s>>>(bt->d_reps, nr, mA, st);
    CR_TRY(launch_check(bt, "column_kernel"));
    next_v_kernel<<<nv, kThreads, 0, s>>>(bt->d_reps, vec, mA, st);
    CR_TRY(launch_check(bt, "next_v_kernel"));
    advance_kernel<<<blocks_of_reps(nr), 128, 0, s>>>(bt->d_reps, nr, mA, st);
    CR_TRY(launch_check(bt, "advance_kernel"));
    ++bt->steps;
    return batch_check(bt, cudaMemcpyAsync(bt->h_state, bt->d_state, (size_t)nr * sizeof(BState),
                                           cudaMemcpyDeviceToHost, s),
                       "state read-back");
}

// End of the cycles of the replicas in the end mask: update x, the FP64 residual of the
// next refinement step (CR_MIXED: rr; CR_FP64: r) and its squared norm.
int batch_cycle_end(cr_batch *bt) {
    const int *mE = mask_ptr(bt, kMaskEnd);
    const int nv = bt->n_items[BL_VEC], nr = bt->n;
    BState *st = reinterpret_cast<BState *>(bt->d_state);
    cudaStream_t s = bt->stream;
    const bool mixed = bt->precision == CR_MIXED;
    cycle_solve_kernel<<<blocks_of_reps(nr), 128, 0, s>>>(bt->d_reps, nr, mE, st);
    CR_TRY(launch_check(bt, "cycle_solve_kernel"));
    update_kernel<<<nv, kThreads, 0, s>>>(bt->d_reps, bt->d_items[BL_VEC], mE, st, mixed ? 1 : 0);
    CR_TRY(launch_check(bt, "update_kernel"));
    const int out = mixed ? BV_RR : BV_R;
    CR_TRY(batch_operator_p(bt, CR_FP64, kMaskEnd, BV_X, out));
    residual_kernel<<<nv, kThreads, 0, s>>>(bt->d_reps, bt->d_items[BL_VEC], mE, out);
    CR_TRY(launch_check(bt, "residual_kernel"));
    CR_TRY(batch_norms(bt, kMaskEnd, out));
    CR_TRY(batch_check(bt, cudaMemcpyAsync(bt->h_norm2, bt->d_norm2, (size_t)nr * sizeof(double),
                                           cudaMemcpyDeviceToHost, s),
                       "norm read-back"));
    return batch_check(bt, cudaStreamSynchronize(s), "cycle end");
}

int upload_masks(cr_batch *bt) {
    return batch_check(bt, cudaMemcpyAsync(bt->d_mask, bt->h_mask, (size_t)4 * bt->n * sizeof(int),
                                           cudaMemcpyHostToDevice, bt->stream),
                       "mask upload");
}
int upload_scal(cr_batch *bt) {
    return batch_check(bt, cudaMemcpyAsync(bt->d_scal, bt->h_scal, (size_t)3 * bt->n * sizeof(double),
                                           cudaMemcpyHostToDevice, bt->stream),
                       "scalar upload");
}

// The next cycle of replica i, or its end (solver.cu's solve/fgmres decisions).
void next_cycle(cr_batch *bt, int i, Run &u, int maxit) {
    const int n = bt->n;
    if (!std::isfinite(u.rnorm)) {
        u.status = CR_NUMERICAL;
        u.phase = kDone;
        return;
    }
    if (u.rnorm <= u.atol || u.s.iterations >= maxit || (bt->precision == CR_MIXED && u.outer >= 20)) {
        u.phase = kDone;
        return;
    }
    double cyc_atol = u.atol;
    if (bt->precision == CR_MIXED) {
        ++u.s.refinements;
        const double want = 0.3 * u.atol / u.rnorm;
        const double inner_rel = std::min(0.5, want >= 1e-4 ? want : 1e-3);
        cyc_atol = inner_rel * u.rnorm;
        if (!(u.rnorm > cyc_atol)) {
            u.phase = kDone;
            return;
        }
    }
    bt->h_scal[i] = 1.0 / u.rnorm;
    bt->h_scal[n + i] = u.rnorm;
    bt->h_scal[2 * n + i] = cyc_atol;
    u.phase = kStart;
}

// Initial residuals of the replicas in `newr` (just set up): ||b||, ||x0||, r0 = b - A64 x0
// (or b from a zero start: A 0 = 0 exactly), CR_MIXED's refinement residual rr = r0, and
// each replica's first cycle.  Uses the all-replica mask slot for the set.
int init_replicas(cr_batch *bt, std::vector<Run> &run, const std::vector<int> &newr) {
    const int n = bt->n;
    int *hm = bt->h_mask;
    std::memset(hm, 0, (size_t)4 * n * sizeof(int));
    for (int i : newr) hm[kMaskAll * n + i] = 1;
    CR_TRY(upload_masks(bt));
    CR_TRY(upload_slot(bt, 0, newr));
    use_slot(bt, 0);
    CR_TRY(batch_norms(bt, kMaskAll, BV_B, 0));
    CR_TRY(batch_norms(bt, kMaskAll, BV_X, n));
    CR_TRY(batch_check(bt, cudaMemcpyAsync(bt->h_norm2, bt->d_norm2, 2 * n * sizeof(double), cudaMemcpyDeviceToHost,
                                           bt->stream),
                       "norm read-back"));
    CR_TRY(batch_check(bt, cudaStreamSynchronize(bt->stream), "norms"));
    for (int i : newr) {
        run[i].bnorm = std::sqrt(std::max(0.0, bt->h_norm2[i]));
        run[i].atol = run[i].tol * run[i].bnorm;
    }
    bool any_x = false;
    for (int i : newr) {
        const bool nz = std::sqrt(std::max(0.0, bt->h_norm2[n + i])) != 0.0;
        hm[kMaskEnd * n + i] = nz ? 1 : 0;    // nonzero starts
        hm[kMaskStart * n + i] = nz ? 0 : 1;  // zero starts
        if (nz) ++run[i].s.matvecs_fp64;
        any_x = any_x || nz;
    }
    CR_TRY(upload_masks(bt));
    copy_kernel<<<bt->n_items[BL_VEC], kThreads, 0, bt->stream>>>(bt->d_reps, bt->d_items[BL_VEC],
                                                                  mask_ptr(bt, kMaskStart), BV_B, BV_R);
    CR_TRY(launch_check(bt, "copy_kernel"));
    if (any_x) {
        CR_TRY(batch_operator_p(bt, CR_FP64, kMaskEnd, BV_X, BV_R));
        residual_kernel<<<bt->n_items[BL_VEC], kThreads, 0, bt->stream>>>(bt->d_reps, bt->d_items[BL_VEC],
                                                                          mask_ptr(bt, kMaskEnd), BV_R);
        CR_TRY(launch_check(bt, "residual_kernel"));
    }
    CR_TRY(batch_norms(bt, kMaskAll, BV_R));
    if (bt->precision == CR_MIXED) {
        copy_kernel<<<bt->n_items[BL_VEC], kThreads, 0, bt->stream>>>(bt->d_reps, bt->d_items[BL_VEC],
                                                                      mask_ptr(bt, kMaskAll), BV_R, BV_RR);
        CR_TRY(launch_check(bt, "copy_kernel"));
    }
    CR_TRY(batch_check(bt, cudaMemcpyAsync(bt->h_norm2, bt->d_norm2, n * sizeof(double), cudaMemcpyDeviceToHost,
                                           bt->stream),
                       "norm read-back"));
    CR_TRY(batch_check(bt, cudaStreamSynchronize(bt->stream), "initial residual"));
    for (int i : newr) {
        Run &u = run[i];
        u.rnorm = std::sqrt(std::max(0.0, bt->h_norm2[i]));
        u.s.initial_residual = u.bnorm > 0 ? u.rnorm / u.bnorm : u.rnorm;
        if (!std::isfinite(u.bnorm)) {
            u.status = CR_NUMERICAL;
            u.phase = kDone;
            continue;
        }
        next_cycle(bt, i, u, u.maxit);
    }
    return CR_OK;
}

// One lockstep round: start the new cycles, one Arnoldi step of every replica in a cycle,
// then the ends of the cycles that finished.  Returns false in *any when no replica took
// part.
int round_once(cr_batch *bt, std::vector<Run> &run, bool *any) {
    const int n = bt->n;
    const int inner = bt->precision == CR_MIXED ? CR_FP32 : CR_FP64;
    int *hm = bt->h_mask;
    bool any_step = false;
    for (int i = 0; i < n; ++i) {
        hm[kMaskStart * n + i] = run[i].phase == kStart;
        if (run[i].phase == kStart) run[i].phase = kArnoldi;
        hm[kMaskStep * n + i] = run[i].phase == kArnoldi;
        hm[kMaskEnd * n + i] = 0;
        hm[kMaskAll * n + i] = 0;
        any_step = any_step || run[i].phase == kArnoldi;
    }
    *any = any_step;
    if (!any_step) return CR_OK;
    CR_TRY(upload_masks(bt));
    CR_TRY(upload_scal(bt));
    // the step's work lists hold only the replicas that take the step
    std::vector<int> set;
    for (int i = 0; i < n; ++i)
        if (hm[kMaskStep * n + i]) set.push_back(i);
    if (set != bt->step_set) {
        CR_TRY(upload_slot(bt, 1, set));
        bt->step_set = set;
    }
    use_slot(bt, 1);
    CR_TRY(batch_step(bt, inner));
    CR_TRY(batch_check(bt, cudaStreamSynchronize(bt->stream), "Arnoldi step"));
    const BState *hs = reinterpret_cast<const BState *>(bt->h_state);
    bool any_end = false;
    for (int i = 0; i < n; ++i) {
        Run &u = run[i];
        if (u.phase != kArnoldi) continue;
        if (inner == CR_FP32) ++u.s.matvecs_fp32;
        else ++u.s.matvecs_fp64;
        if (hs[i].stop == 2) {
            u.status = CR_NUMERICAL;
            u.phase = kDone;
            continue;
        }
        if (hs[i].frozen || u.s.iterations + hs[i].j >= u.maxit) {
            u.phase = kEnd;
            hm[kMaskEnd * n + i] = 1;
            any_end = true;
        }
    }
    if (!any_end) return CR_OK;
    std::vector<int> ends;
    for (int i = 0; i < n; ++i) {
        hm[kMaskStep * n + i] = hm[kMaskStart * n + i] = 0;
        if (hm[kMaskEnd * n + i]) ends.push_back(i);
    }
    CR_TRY(upload_masks(bt));
    CR_TRY(upload_slot(bt, 0, ends));
    use_slot(bt, 0);
    CR_TRY(batch_cycle_end(bt));
    for (int i = 0; i < n; ++i) {
        Run &u = run[i];
        if (u.phase != kEnd) continue;
        u.s.iterations += hs[i].j;
        ++u.s.restarts;
        ++u.s.matvecs_fp64;
        ++u.outer;
        u.rnorm = std::sqrt(std::max(0.0, bt->h_norm2[i]));
        next_cycle(bt, i, u, u.maxit);
    }
    return CR_OK;
}

// Host threads with one stream each, running per-replica tasks (set-up, force pass) from
// a queue while the calling thread runs the lockstep rounds.
class TaskPool {
public:
    typedef std::function<void(int, cr_handle *)> Fn;
    // The task streams take the highest priority: a set-up is a latency-bound chain of
    // small kernels that the rounds' full-GPU kernels would otherwise hold back, delaying
    // the replica's join; the rounds fill the multiprocessors the chains leave free.
    TaskPool(cr_batch *bt, int threads) : bt_(bt) {
        cudaGetDevice(&dev_);
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        for (int t = 0; t < threads; ++t) {
            cudaStream_t s = nullptr;
            if (cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, greatest) != cudaSuccess) {
                cudaGetLastError();
                break;
            }
            streams_.push_back(s);
        }
        for (size_t t = 0; t < streams_.size(); ++t) threads_.emplace_back([this, t] { work(t); });
    }
    ~TaskPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &th : threads_) th.join();
        for (cudaStream_t s : streams_) cudaStreamDestroy(s);
    }
    bool ok() const { return !streams_.empty(); }
    void push(int i, Fn f) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back({i, std::move(f)});
            ++pending_;
        }
        cv_.notify_one();
    }
    // Replicas whose tasks finished since the last call (waits up to `wait_ms` for one when
    // `block` is set and none is there yet).
    std::vector<int> finished(bool block) {
        std::unique_lock<std::mutex> lk(mu_);
        if (block && done_.empty() && pending_ > 0) done_cv_.wait(lk, [this] { return !done_.empty() || pending_ == 0; });
        std::vector<int> out;
        out.swap(done_);
        return out;
    }
    int pending() {
        std::lock_guard<std::mutex> lk(mu_);
        return pending_;
    }
    void drain() {
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return pending_ == 0; });
    }

private:
    struct Task {
        int i;
        Fn f;
    };
    void work(size_t t) {
        cudaSetDevice(dev_);
        for (;;) {
            Task task;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;
                task = std::move(q_.front());
                q_.pop_front();
            }
            cr_handle *h = bt_->handles[task.i];
            cudaStream_t saved = h->stream;
            h->stream = streams_[t];
            task.f(task.i, h);
            cudaStreamSynchronize(streams_[t]);
            h->stream = saved;
            {
                std::lock_guard<std::mutex> lk(mu_);
                done_.push_back(task.i);
                --pending_;
            }
            done_cv_.notify_all();
        }
    }
    cr_batch *bt_;
    int dev_ = 0;
    std::vector<cudaStream_t> streams_;
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::deque<Task> q_;
    std::vector<int> done_;
    int pending_ = 0;
    bool stop_ = false;
};

// Requirements every member handle meets for the batched kernels (checked at creation
// and before every solve).
int check_member(cr_batch *bt, int i, cr_handle *h) {
    const std::string who = "lockstep batch: replica " + std::to_string(i) + ": ";
    if (!h) return batch_fail(bt, CR_BAD_PARAM, who + "null handle");
    if (!h->have_topology) return batch_fail(bt, CR_NOT_READY, who + "topology not set");
    if (h->user.precision != bt->precision) return batch_fail(bt, CR_BAD_PARAM, who + "precision differs");
    if (h->user.precond != bt->precond) return batch_fail(bt, CR_BAD_PARAM, who + "preconditioner differs");
    if (h->kry.m != bt->m) return batch_fail(bt, CR_BAD_PARAM, who + "restart length differs");
    if (h->d.support != bt->support) return batch_fail(bt, CR_BAD_PARAM, who + "support differs");
    if (h->tile != 8 || h->spread_mode != 0)
        return batch_fail(bt, CR_BAD_PARAM, who + "mesh tiling must be 8^3 tiles with register-column spreading");
    if (h->user.learned || h->corr.net)
        return batch_fail(bt, CR_BAD_PARAM, who + "the learned start and correction are single-system features");
    if (h->rs_onfly & (CR_REALSPACE_ONFLY32 | CR_REALSPACE_ONFLY64 | CR_REALSPACE_STREAM))
        return batch_fail(bt, CR_BAD_PARAM, who + "real space must use stored values and the direct product");
    const double *chk = bt->h_grid_check.data() + (size_t)6 * i;
    for (int d = 0; d < 3; ++d)
        if (chk[d] != h->d.grid[d] || chk[3 + d] != h->L[d])
            return batch_fail(bt, CR_BAD_PARAM, who + "mesh or box changed since the batch was created");
    return CR_OK;
}

void destroy_batch(cr_batch *bt) {
    for (BatchFftGroup &G : bt->groups)
        for (int p = 0; p < 2; ++p) {
            if (G.fwd[p]) cufftDestroy(G.fwd[p]);
            if (G.inv[p]) cufftDestroy(G.inv[p]);
        }
    for (void *p : {(void *)bt->d_reps, (void *)bt->slot_base[0], (void *)bt->slot_base[1], (void *)bt->d_mask,
                    (void *)bt->grid32,
                    (void *)bt->scale32, (void *)bt->grid64, (void *)bt->scale64, (void *)bt->spec32,
                    (void *)bt->spec64, bt->d_state, (void *)bt->d_norm2, (void *)bt->d_scal})
        if (p) cudaFree(p);
    for (void *p : {(void *)bt->h_mask, bt->h_state, (void *)bt->h_norm2, (void *)bt->h_scal,
                    (void *)bt->pin_items[0], (void *)bt->pin_items[1]})
        if (p) cudaFreeHost(p);
    for (cudaEvent_t e : {bt->ev_fork, bt->ev_join, bt->ev0, bt->ev1})
        if (e) cudaEventDestroy(e);
    if (bt->stream) cudaStreamDestroy(bt->stream);
    if (bt->side) cudaStreamDestroy(bt->side);
    delete bt;
}

int create_batch(cr_batch *bt, int n, cr_handle *const *handles) {
    bt->n = n;
    bt->handles.assign(handles, handles + n);
    cr_handle *h0 = handles[0];
    if (!h0) return batch_fail(bt, CR_BAD_PARAM, "lockstep batch: null handle");
    bt->precision = h0->user.precision;
    bt->precond = h0->user.precond;
    bt->m = h0->kry.m;
    bt->support = h0->d.support;
    if (bt->precision != CR_MIXED && bt->precision != CR_FP64)
        return batch_fail(bt, CR_BAD_PARAM, "lockstep batch: precision must be CR_MIXED or CR_FP64");
    if (bt->support != 9 && bt->support != 11)
        return batch_fail(bt, CR_BAD_PARAM, "lockstep batch: support must be 9 or 11");
    bt->h_grid_check.assign((size_t)6 * n, 0.0);
    for (int i = 0; i < n; ++i) {
        cr_handle *h = handles[i];
        if (!h) return batch_fail(bt, CR_BAD_PARAM, "lockstep batch: null handle");
        for (int d = 0; d < 3; ++d) {
            bt->h_grid_check[(size_t)6 * i + d] = h->d.grid[d];
            bt->h_grid_check[(size_t)6 * i + 3 + d] = h->L[d];
        }
        CR_TRY(check_member(bt, i, h));
    }
    // size groups, in order of first appearance
    std::map<std::tuple<int, int, int>, int> gidx;
    bt->rep_group.assign(n, 0);
    for (int i = 0; i < n; ++i) {
        const auto key = std::make_tuple(handles[i]->d.grid[0], handles[i]->d.grid[1], handles[i]->d.grid[2]);
        auto f = gidx.find(key);
        if (f == gidx.end()) {
            f = gidx.emplace(key, (int)bt->groups.size()).first;
            BatchFftGroup G;
            for (int d = 0; d < 3; ++d) G.grid[d] = handles[i]->d.grid[d];
            bt->groups.push_back(G);
        }
        bt->rep_group[i] = f->second;
        bt->groups[f->second].reps.push_back(i);
    }
    // every group starts on a 256-byte boundary of the mesh and spectrum buffers (cuFFT
    // wants its pointers aligned; an odd-sized mesh before a group would misalign it)
    long long G = 0, S = 0;
    for (BatchFftGroup &g : bt->groups) {
        G = (G + 63) / 64 * 64;
        S = (S + 15) / 16 * 16;
        g.goff = G;
        g.soff = S;
        const long long gn = (long long)g.grid[0] * g.grid[1] * g.grid[2];
        const long long sn = (long long)g.grid[0] * g.grid[1] * (g.grid[2] / 2 + 1);
        G += gn * (long long)g.reps.size();
        S += sn * (long long)g.reps.size();
    }
    if (S >= (1LL << 31) || G >= (1LL << 31))
        return batch_fail(bt, CR_BAD_PARAM, "lockstep batch: the replicas' meshes exceed 2^31 nodes");
    bt->G = G;
    bt->S = S;
    // rounds at the lowest priority (the per-replica tasks take the highest); the wave part
    // one level above the real-space product beside it, where the device has the levels
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    CR_TRY(batch_check(bt, cudaStreamCreateWithPriority(&bt->stream, cudaStreamNonBlocking, lo), "stream"));
    CR_TRY(batch_check(bt, cudaStreamCreateWithPriority(&bt->side, cudaStreamNonBlocking, lo > hi ? lo - 1 : lo),
                       "stream"));
    for (cudaEvent_t *e : {&bt->ev_fork, &bt->ev_join})
        CR_TRY(batch_check(bt, cudaEventCreateWithFlags(e, cudaEventDisableTiming), "event"));
    for (cudaEvent_t *e : {&bt->ev0, &bt->ev1}) CR_TRY(batch_check(bt, cudaEventCreate(e), "event"));
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->grid32, std::max<long long>(G, 1) * sizeof(float)), "batch mesh"));
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->grid64, std::max<long long>(G, 1) * sizeof(double)), "batch mesh"));
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->spec32, std::max<long long>(S, 1) * sizeof(cufftComplex)),
                       "batch spectrum"));
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->spec64, std::max<long long>(S, 1) * sizeof(cufftDoubleComplex)),
                       "batch spectrum"));
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->scale32, std::max<long long>(S, 1) * sizeof(float)),
                       "batch influence function"));
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->scale64, std::max<long long>(S, 1) * sizeof(double)),
                       "batch influence function"));
    // every replica's influence function at its place in the batch spectrum
    for (BatchFftGroup &g : bt->groups) {
        const long long sn = (long long)g.grid[0] * g.grid[1] * (g.grid[2] / 2 + 1);
        for (size_t q = 0; q < g.reps.size(); ++q) {
            const cr_handle *h = handles[g.reps[q]];
            const long long off = g.soff + (long long)q * sn;
            CR_TRY(batch_check(bt, cudaMemcpyAsync(bt->scale32 + off, h->m32.scale, sn * sizeof(float),
                                                   cudaMemcpyDeviceToDevice, bt->stream),
                               "influence function copy"));
            CR_TRY(batch_check(bt, cudaMemcpyAsync(bt->scale64 + off, h->m64.scale, sn * sizeof(double),
                                                   cudaMemcpyDeviceToDevice, bt->stream),
                               "influence function copy"));
        }
        int dims[3] = {g.grid[0], g.grid[1], g.grid[2]};
        const int cnt = (int)g.reps.size();
        if (cufftPlanMany(&g.fwd[0], 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, cnt) != CUFFT_SUCCESS ||
            cufftPlanMany(&g.inv[0], 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, cnt) != CUFFT_SUCCESS ||
            cufftPlanMany(&g.fwd[1], 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, cnt) != CUFFT_SUCCESS ||
            cufftPlanMany(&g.inv[1], 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, cnt) != CUFFT_SUCCESS)
            return batch_fail(bt, CR_CUDA_ERROR, "lockstep batch: batched cuFFT plan creation failed");
    }
    bt->reps.assign(n, BatchRep{});
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->d_reps, (size_t)n * sizeof(BatchRep)), "descriptors"));
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->d_mask, (size_t)4 * n * sizeof(int)), "masks"));
    CR_TRY(batch_check(bt, cudaMallocHost((void **)&bt->h_mask, (size_t)4 * n * sizeof(int)), "masks"));
    CR_TRY(batch_check(bt, cudaMalloc(&bt->d_state, (size_t)n * sizeof(BState)), "states"));
    CR_TRY(batch_check(bt, cudaMallocHost(&bt->h_state, (size_t)n * sizeof(BState)), "states"));
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->d_norm2, (size_t)2 * n * sizeof(double)), "norms"));
    CR_TRY(batch_check(bt, cudaMallocHost((void **)&bt->h_norm2, (size_t)2 * n * sizeof(double)), "norms"));
    CR_TRY(batch_check(bt, cudaMalloc((void **)&bt->d_scal, (size_t)3 * n * sizeof(double)), "scalars"));
    CR_TRY(batch_check(bt, cudaMallocHost((void **)&bt->h_scal, (size_t)3 * n * sizeof(double)), "scalars"));
    std::memset(bt->h_scal, 0, (size_t)3 * n * sizeof(double));
    CR_TRY(batch_check(bt, cudaMemsetAsync(bt->d_state, 0, (size_t)n * sizeof(BState), bt->stream), "states"));
    CR_TRY(batch_mesh_attrs(bt));
    return batch_check(bt, cudaStreamSynchronize(bt->stream), "batch creation");
}

}  // namespace
}  // namespace cr

using namespace cr;

extern "C" {

static thread_local std::string g_create_error;

int cr_batch_create(int n, cr_handle *const *handles, cr_batch **out) {
    g_create_error.clear();
    if (!out) return CR_BAD_PARAM;
    *out = nullptr;
    if (n <= 0 || !handles) {
        g_create_error = "lockstep batch: no handles";
        return CR_BAD_PARAM;
    }
    cr_batch *bt = new cr_batch();
    const int st = create_batch(bt, n, handles);
    if (st != CR_OK) {
        g_create_error = bt->last_error;
        destroy_batch(bt);
        return st;
    }
    *out = bt;
    return CR_OK;
}

int cr_batch_destroy(cr_batch *bt) {
    if (!bt) return CR_BAD_PARAM;
    destroy_batch(bt);
    return CR_OK;
}

const char *cr_batch_last_error(const cr_batch *bt) { return bt ? bt->last_error.c_str() : g_create_error.c_str(); }

int cr_batch_phase_ms(const cr_batch *bt, double *first_join_ms, double *rounds_ms, double *total_ms) {
    if (!bt) return CR_BAD_PARAM;
    if (first_join_ms) *first_join_ms = bt->phase_ms[0];
    if (rounds_ms) *rounds_ms = bt->phase_ms[1];
    if (total_ms) *total_ms = bt->phase_ms[2];
    return CR_OK;
}

int cr_batch_counters(const cr_batch *bt, long long *kernel_launches, long long *fft_execs, long long *steps) {
    if (!bt) return CR_BAD_PARAM;
    if (kernel_launches) *kernel_launches = bt->launches;
    if (fft_execs) *fft_execs = bt->fft_execs;
    if (steps) *steps = bt->steps;
    return CR_OK;
}

int cr_batch_solve(cr_batch *bt, const double *const *d_pos, const double *const *d_body_pos, double *const *d_q,
                   double *const *d_phi, double *const *d_force, cr_solve_stats *stats, int *status, int n_threads) {
    if (!bt || bt->n <= 0 || !bt->stream) return CR_BAD_PARAM;
    const int n = bt->n;
    if (!d_pos || !d_body_pos || !d_q || !d_phi || !d_force || !status)
        return batch_fail(bt, CR_BAD_PARAM, "lockstep batch: null argument array");
    for (int i = 0; i < n; ++i) {
        CR_TRY(check_member(bt, i, bt->handles[i]));
        const cr_handle *h = bt->handles[i];
        if (h->N > 0 && (!d_pos[i] || !d_q[i] || !d_force[i]))
            return batch_fail(bt, CR_BAD_PARAM, "lockstep batch: null array of replica " + std::to_string(i));
        if (h->B > 0 && (!d_phi[i] || !d_body_pos[i]))
            return batch_fail(bt, CR_BAD_PARAM, "lockstep batch: null body array of replica " + std::to_string(i));
    }
    bt->last_error.clear();
    using clock = std::chrono::steady_clock;
    auto ms_since = [](clock::time_point t) {
        return std::chrono::duration<double, std::milli>(clock::now() - t).count();
    };
    const clock::time_point t0 = clock::now();
    bt->phase_ms[0] = bt->phase_ms[1] = bt->phase_ms[2] = 0.0;
    std::vector<Run> run(n);
    for (int i = 0; i < n; ++i) {
        const cr_handle *h = bt->handles[i];
        run[i].tol = h->user.gmres_tol > 0 ? h->user.gmres_tol : h->user.errortol;
        run[i].maxit = h->user.maxiter > 0 ? h->user.maxiter : 100;
        status[i] = CR_OK;
    }
    bt->cond_threads = 64;
    bt->cond_smem = 0;
    bt->model_smem = 0;
    for (int k = 0; k < BL_COUNT; ++k) {
        bt->h_full[k].clear();
        bt->rep_range[k].assign(2 * (size_t)n, 0);
        bt->n_items[k] = 0;
    }
    bt->step_set.clear();
    Shapes shapes;
    const bool mixed = bt->precision == CR_MIXED;
    // Per-replica tasks: the set-up of every replica (largest first) and, once it has
    // converged, its force pass.  status[i] is written by the task's thread only.
    auto setup = [&](int i, cr_handle *h) {
        int st = geometry_update(h, d_pos[i], d_body_pos[i]);
        Krylov &K = h->kry;
        if (st == CR_OK) st = objective(h, K.b);
        if (st == CR_OK)
            st = check_cuda(h, cudaMemcpyAsync(K.x, d_q[i], h->N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream),
                            "start copy");
        if (st == CR_OK && h->B)
            st = check_cuda(h, cudaMemcpyAsync(K.x + h->N, d_phi[i], h->B * sizeof(double), cudaMemcpyDeviceToDevice,
                                               h->stream),
                            "start copy");
        if (st == CR_OK && mixed) st = realspace_prepare(h, CR_FP32);
        if (st == CR_OK) st = realspace_prepare(h, CR_FP64);
        if (st == CR_OK) st = coarse_prepare(h);
        if (st == CR_OK && bt->precond != CR_PRECOND_DIAGONAL && h->B > 0 && !h->cond.ready)
            st = fail(h, CR_NOT_READY, "conductor preconditioner not set up");
        status[i] = st;
    };
    auto forces = [&](int i, cr_handle *h) {
        int st = check_cuda(h, cudaMemcpyAsync(d_q[i], h->kry.x, h->N * sizeof(double), cudaMemcpyDeviceToDevice,
                                               h->stream),
                            "solution copy");
        if (st == CR_OK && h->B)
            st = check_cuda(h, cudaMemcpyAsync(d_phi[i], h->kry.x + h->N, h->B * sizeof(double),
                                               cudaMemcpyDeviceToDevice, h->stream),
                            "solution copy");
        if (st == CR_OK) st = cast_charges(h, h->m64, h->kry.x);
        if (st == CR_OK) st = wave_force(h, h->m64);
        if (st == CR_OK) st = real_space_force(h, h->m64, h->kry.x, d_force[i]);
        status[i] = st;
    };
    std::vector<int> order;
    for (int i = 0; i < n; ++i) {
        if (bt->handles[i]->N == 0) {
            run[i].phase = kDone;
            run[i].s.converged = 1;
        } else {
            order.push_back(i);
        }
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return bt->handles[a]->N + bt->handles[a]->B > bt->handles[b]->N + bt->handles[b]->B;
    });
    int err = CR_OK;
    std::vector<char> in_setup(n, 0), in_force(n, 0);
    {
        TaskPool pool(bt, std::max(1, std::min((int)std::max<size_t>(order.size(), 1), n_threads > 0 ? n_threads : 16)));
        if (!pool.ok()) return batch_fail(bt, CR_CUDA_ERROR, "lockstep batch: no worker stream");
        for (int i : order) {
            in_setup[i] = 1;
            pool.push(i, setup);
        }
        std::vector<int> live;
        bool started = false;
        double first_join_ms = -1.0;
        // rounds: replicas join once set up, leave for their force pass once converged
        for (;;) {
            bool active = false;
            for (int i = 0; i < n; ++i) active = active || (run[i].phase >= kStart && run[i].phase <= kEnd);
            std::vector<int> fin = pool.finished(!active);
            std::vector<int> joined;
            for (int i : fin) {
                if (in_setup[i]) {
                    in_setup[i] = 0;
                    if (status[i] != CR_OK) {
                        run[i].status = status[i];
                        run[i].phase = kDone;
                    } else if (err == CR_OK) {
                        err = describe_rep(bt, i, shapes);
                        if (err == CR_OK) joined.push_back(i);
                    }
                } else if (in_force[i]) {
                    in_force[i] = 0;
                }
            }
            if (err != CR_OK) break;
            if (!joined.empty()) {
                if (!started) {
                    started = true;
                    first_join_ms = ms_since(t0);
                    err = batch_check(bt, cudaEventRecord(bt->ev0, bt->stream), "event");
                    if (err != CR_OK) break;
                }
                live.insert(live.end(), joined.begin(), joined.end());
                err = publish(bt, joined);
                if (err == CR_OK) err = init_replicas(bt, run, joined);
                if (err != CR_OK) break;
            }
            bool any = false;
            err = round_once(bt, run, &any);
            if (err != CR_OK) break;
            // finished replicas leave for their force pass (also when not converged, as
            // cr_compute does; not after a numerical failure)
            for (int i : live)
                if (run[i].phase == kDone && !run[i].force_queued) {
                    run[i].force_queued = true;
                    if (run[i].status == CR_OK) {
                        in_force[i] = 1;
                        pool.push(i, forces);
                    }
                }
            if (!any && pool.pending() == 0) {
                bool waiting = false;
                for (int i = 0; i < n; ++i) waiting = waiting || in_setup[i] || in_force[i];
                if (!waiting) break;
            }
        }
        pool.drain();
        for (int i : pool.finished(false))
            if (in_force[i]) in_force[i] = 0;
        bt->phase_ms[0] = first_join_ms;
    }
    if (err != CR_OK) return err;
    float loop_ms = 0.f;
    bool any_live = false;
    for (int i = 0; i < n; ++i) any_live = any_live || bt->handles[i]->N > 0;
    if (any_live && bt->phase_ms[0] >= 0.0) {
        CR_TRY(batch_check(bt, cudaEventRecord(bt->ev1, bt->stream), "event"));
        CR_TRY(batch_check(bt, cudaStreamSynchronize(bt->stream), "batch solve"));
        if (cudaEventElapsedTime(&loop_ms, bt->ev0, bt->ev1) != cudaSuccess) {
            cudaGetLastError();
            loop_ms = 0.f;
        }
    }
    bt->phase_ms[1] = loop_ms;
    bt->phase_ms[2] = ms_since(t0);
    int worst = CR_OK;
    for (int i = 0; i < n; ++i) {
        Run &u = run[i];
        if (u.force_queued && u.status == CR_OK && status[i] != CR_OK) u.status = status[i];  // force pass failed
        if (bt->handles[i]->N > 0 && u.status == CR_OK) {
            u.s.final_residual = u.bnorm > 0 ? u.rnorm / u.bnorm : u.rnorm;
            u.s.converged = u.rnorm <= u.atol ? 1 : 0;
            if (!u.s.converged) u.status = CR_NOT_CONVERGED;
        }
        u.s.solve_ms = loop_ms;
        if (stats) stats[i] = u.s;
        status[i] = u.status;
        if (status[i] != CR_OK && (worst == CR_OK || worst == CR_NOT_CONVERGED)) worst = status[i];
    }
    if (worst != CR_OK && bt->last_error.empty()) bt->last_error = "lockstep batch: a replica failed (see status)";
    return worst;
}

}  // extern "C"
