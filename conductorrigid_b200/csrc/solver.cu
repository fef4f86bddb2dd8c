// solver.cu -- matrix-free flexible GMRES for the saddle-point system.
//
// Replaces the reference's cusp::krylov::gmres(M, q, rhs, 10, monitor, Pr) call
// (ConductorRigid.cu:1134-1136): restarted GMRES with the same diagonal
// preconditioner and warm start.  Differences, all of which leave the fixed point
// A x = b untouched:
//   - the preconditioner is applied on the right (flexible GMRES, so a varying
//     preconditioner such as the learned correction is allowed), and convergence is
//     judged on the true residual ||b - A x|| <= tol ||b|| recomputed with the FP64
//     operator, where CUSP stops on the left-preconditioned residual;
//   - the Krylov basis, Gram-Schmidt dot products (classical Gram-Schmidt with one
//     reorthogonalisation), Givens rotations and the least-squares update are FP64;
//   - CR_MIXED runs the inner iterations with the FP32 operator and wraps them in
//     FP64 iterative refinement: r = b - A64 x, solve A32 d ~= r, x += d.
// All vectors stay on the device.  An uncaptured Arnoldi step copies its Hessenberg
// column to pinned host memory for the Givens update; a captured step (below) does that
// update on the device and copies back only its small state.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cr_internal.cuh"

namespace cr {

namespace {

constexpr int kDotThreads = 256;

// partial[blk * kmax + j] = sum over this block's rows of V_j[i] * w[i]   (j < k):
// eight vectors per pass, so w is read once and the block reduces once per eight.
constexpr int kDotChunk = 8;
__device__ __forceinline__ void multi_dot_body(int n, int k, int kmax, const double *__restrict__ V,
                                               const double *__restrict__ w, double *__restrict__ partial) {
    __shared__ double red[kDotThreads / 32][kDotChunk];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j0 = 0; j0 < k; j0 += kDotChunk) {
        double acc[kDotChunk];
#pragma unroll
        for (int c = 0; c < kDotChunk; ++c) acc[c] = 0.0;
        const int kc = min(kDotChunk, k - j0);
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            const double wi = w[i];
#pragma unroll
            for (int c = 0; c < kDotChunk; ++c)
                if (c < kc) acc[c] += V[(size_t)(j0 + c) * n + i] * wi;
        }
#pragma unroll
        for (int c = 0; c < kDotChunk; ++c) {
            for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
            if (lane == 0) red[warp][c] = acc[c];
        }
        __syncthreads();
        if (threadIdx.x < kc) {
            double t = 0.0;
            for (int q = 0; q < kDotThreads / 32; ++q) t += red[q][threadIdx.x];
            partial[(size_t)blockIdx.x * kmax + j0 + threadIdx.x] = t;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kDotThreads) multi_dot_kernel(int n, int k, const double *__restrict__ V,
                                                                const double *__restrict__ w,
                                                                double *__restrict__ partial) {
    multi_dot_body(n, k, k, V, w, partial);
}

// out[j] = sum_blk partial[blk * k + j], in block order (deterministic).
__global__ void reduce_partials_kernel(int nblk, int k, const double *__restrict__ partial, double *__restrict__ out) {
    const int j = blockIdx.x;
    const int lane = threadIdx.x;
    double s = 0.0;
    for (int b = lane; b < nblk; b += 32) s += partial[(size_t)b * k + j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[j] = s;
}

// w -= sum_j h[j] V_j
__global__ void project_kernel(int n, int k, const double *__restrict__ V, const double *__restrict__ hv,
                               double *__restrict__ w) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = w[i];
#pragma unroll 8
        for (int j = 0; j < k; ++j) s -= hv[j] * V[(size_t)j * n + i];
        w[i] = s;
    }
}

__global__ void scale_kernel(int n, double a, const double *__restrict__ x, double *__restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a * x[i];
}

// y = b - y
__global__ void residual_kernel(int n, const double *__restrict__ b, double *__restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = b[i] - y[i];
}

// x += sum_j c[j] Z_j
__global__ void update_kernel(int n, int k, const double *__restrict__ Z, const double *__restrict__ c,
                              double *__restrict__ x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = x[i];
        for (int j = 0; j < k; ++j) s += c[j] * Z[(size_t)j * n + i];
        x[i] = s;
    }
}

__global__ void axpy_kernel(int n, double a, const double *__restrict__ x, double *__restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += a * x[i];
}

// ---- captured Arnoldi step --------------------------------------------------------
// With a stream set and the profiler off, one Arnoldi step is captured once per geometry
// as a CUDA graph and launched once per iteration.  Everything that depends on the
// column index lives in device memory (ArnoldiState), so one graph serves every step:
// V_j and Z_j pass through fixed staging vectors, the dot/projection kernels read their
// length from the state, and the Hessenberg column, the Givens rotations and the
// stopping test run in a one-thread kernel.  The last node copies the state to pinned
// host memory, which the host reads after each launch to stop exactly where the eager
// loop would.
struct ArnoldiState {
    int j;          // columns completed in this cycle
    int stop;       // 1: the last column met the tolerance or broke down; 2: non-finite norm
    int frozen;     // set once a stopping column is counted: later launches change nothing
    int pad;
    double res;     // |g[j]| after the last counted column
    double inv_hn;  // 1 / ||w|| of the column being added
    double atol;    // absolute tolerance of this cycle
};

__global__ void init_cycle_kernel(int m, double beta, double atol, ArnoldiState *st, double *__restrict__ g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= m) g[i] = i == 0 ? beta : 0.0;
    if (i == 0) {
        st->j = 0;
        st->stop = 0;
        st->frozen = 0;
        st->pad = 0;
        st->res = beta;
        st->inv_hn = 0.0;
        st->atol = atol;
    }
}

__global__ void gather_col_kernel(int n, const double *__restrict__ base, const ArnoldiState *st,
                                  double *__restrict__ dst) {
    const size_t off = (size_t)st->j * n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = base[off + i];
}

__global__ void scatter_col_kernel(int n, int m, const double *__restrict__ src, const ArnoldiState *st,
                                   double *__restrict__ base) {
    const int j = st->j;
    if (j >= m) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        base[(size_t)j * n + i] = src[i];
}

// multi_dot_kernel with k = j + 1 read from the state (at most kmax)
__global__ void __launch_bounds__(kDotThreads) multi_dot_dev_kernel(int n, int kmax, const ArnoldiState *st,
                                                                    const double *__restrict__ V,
                                                                    const double *__restrict__ w,
                                                                    double *__restrict__ partial) {
    multi_dot_body(n, min(st->j + 1, kmax), kmax, V, w, partial);
}

__global__ void reduce_partials_dev_kernel(int nblk, int kmax, const ArnoldiState *st,
                                           const double *__restrict__ partial, double *__restrict__ out) {
    const int j = blockIdx.x;
    if (j >= min(st->j + 1, kmax)) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += 32) s += partial[(size_t)b * kmax + j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[j] = s;
}

__global__ void project_dev_kernel(int n, int kmax, const ArnoldiState *st, const double *__restrict__ V,
                                   const double *__restrict__ hv, double *__restrict__ w) {
    const int k = min(st->j + 1, kmax);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = w[i];
#pragma unroll 8
        for (int j = 0; j < k; ++j) s -= hv[j] * V[(size_t)j * n + i];
        w[i] = s;
    }
}

// The host loop's Hessenberg update for column j, on the device (one thread).
__global__ void arnoldi_column_kernel(int m, ArnoldiState *st, const double *__restrict__ hcol, double *__restrict__ H,
                                      double *__restrict__ cs, double *__restrict__ sn, double *__restrict__ g) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    st->inv_hn = 0.0;
    if (st->frozen) return;
    const int j = st->j;
    if (j >= m) return;
    const double *h1 = hcol, *h2 = hcol + (m + 1);
    const double hn = sqrt(fmax(0.0, hcol[2 * (m + 1)]));
    if (!isfinite(hn)) {
        st->stop = 2;
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
    st->res = fabs(g[j + 1]);
    st->inv_hn = hn > 0 ? 1.0 / hn : 0.0;
    if (fabs(g[j + 1]) <= st->atol || hn == 0.0) st->stop = 1;
}

__global__ void scale_next_kernel(int n, int m, const ArnoldiState *st, const double *__restrict__ w,
                                  double *__restrict__ V) {
    const int j = st->j;
    const double a = st->inv_hn;
    if (st->frozen || j >= m || a == 0.0) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        V[(size_t)(j + 1) * n + i] = a * w[i];
}

__global__ void advance_kernel(int m, ArnoldiState *st) {
    if (blockIdx.x != 0 || threadIdx.x != 0 || st->frozen) return;
    if (st->stop == 2) {
        st->frozen = 1;
        return;
    }
    st->j += 1;
    if (st->stop || st->j >= m) st->frozen = 1;
}

// Learned-guess refit of the body potentials: Phi_b += mean of the bead residuals of
// body b, which zeroes that mean (a bead row is Phi_b - (M q)_i = b_i; the charge rows
// do not involve Phi).  Exact, no operator application.
__global__ void phi_refit_kernel(int N, int B, const int *__restrict__ start, const int *__restrict__ members,
                                 double *__restrict__ x, double *__restrict__ r) {
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= B) return;
    const int k0 = start[b], k1 = start[b + 1];
    double s = 0.0;
    for (int k = k0 + lane; k < k1; k += 32) s += r[members[k]];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double mean = s / (double)(k1 - k0);
    for (int k = k0 + lane; k < k1; k += 32) r[members[k]] -= mean;
    if (lane == 0) x[N + b] += mean;
}

int vec_blocks(int n) { return std::max(1, std::min(4 * 148, blocks_for(n, 256))); }

}  // namespace

// out[0..k) = V[0..k)^T w over the n = N + B unknowns (device result, fixed sum order)
int dots(cr_handle *h, int k, const double *V, const double *w, double *out) {
    ProfScope ps(h, PROF_KRYLOV);
    Krylov &K = h->kry;
    multi_dot_kernel<<<K.nblocks, kDotThreads, 0, h->stream>>>(K.n, k, V, w, K.partial);
    CR_LAUNCH(h, "multi_dot_kernel");
    reduce_partials_kernel<<<k, 32, 0, h->stream>>>(K.nblocks, k, K.partial, out);
    CR_LAUNCH(h, "reduce_partials_kernel");
    return CR_OK;
}

namespace {

int norm(cr_handle *h, const double *v, double *result) {
    Krylov &K = h->kry;
    CR_TRY(dots(h, 1, v, v, K.hcol));
    CR_CUDA(h, cudaMemcpyAsync(K.h_pinned, K.hcol, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    *result = std::sqrt(std::max(0.0, K.h_pinned[0]));
    return CR_OK;
}

struct OpCount {
    int fp64 = 0, fp32 = 0;
};

int op_apply(cr_handle *h, int precision, const double *x, double *y, OpCount &oc) {
    if (precision == CR_FP64) ++oc.fp64;
    else ++oc.fp32;
    return apply_operator(h, x, y, precision);
}

bool graph_mode(const cr_handle *h) { return h->use_graphs && h->stream != nullptr && !h->prof.on; }

// The kernels of one Arnoldi step on the device state (recorded into a graph).
int record_step(cr_handle *h, int precision) {
    Krylov &K = h->kry;
    const int n = K.n, m = K.m, nb = vec_blocks(n);
    cudaStream_t s = h->stream;
    ArnoldiState *st = reinterpret_cast<ArnoldiState *>(K.state);
    OpCount none;
    gather_col_kernel<<<nb, 256, 0, s>>>(n, K.V, st, K.sin);
    CR_LAUNCH(h, "gather_col_kernel");
    CR_TRY(precondition_step(h, K.sin, K.sz));
    scatter_col_kernel<<<nb, 256, 0, s>>>(n, m, K.sz, st, K.Z);
    CR_LAUNCH(h, "scatter_col_kernel");
    CR_TRY(op_apply(h, precision, K.sz, K.w, none));
    for (int pass = 0; pass < 2; ++pass) {  // classical Gram-Schmidt, twice
        double *hv = K.hcol + (size_t)pass * (m + 1);
        multi_dot_dev_kernel<<<K.nblocks, kDotThreads, 0, s>>>(n, m + 1, st, K.V, K.w, K.partial);
        CR_LAUNCH(h, "multi_dot_dev_kernel");
        reduce_partials_dev_kernel<<<m + 1, 32, 0, s>>>(K.nblocks, m + 1, st, K.partial, hv);
        CR_LAUNCH(h, "reduce_partials_dev_kernel");
        project_dev_kernel<<<nb, 256, 0, s>>>(n, m + 1, st, K.V, hv, K.w);
        CR_LAUNCH(h, "project_dev_kernel");
    }
    CR_TRY(dots(h, 1, K.w, K.w, K.hcol + 2 * (m + 1)));
    arnoldi_column_kernel<<<1, 32, 0, s>>>(m, st, K.hcol, K.H, K.cs, K.sn, K.g);
    CR_LAUNCH(h, "arnoldi_column_kernel");
    scale_next_kernel<<<nb, 256, 0, s>>>(n, m, st, K.w, K.V);
    CR_LAUNCH(h, "scale_next_kernel");
    advance_kernel<<<1, 32, 0, s>>>(m, st);
    CR_LAUNCH(h, "advance_kernel");
    CR_CUDA(h, cudaMemcpyAsync(K.h_state, K.state, sizeof(ArnoldiState), cudaMemcpyDeviceToHost, s));
    return CR_OK;
}

// Capture the step for this geometry and operator precision (once per geometry; an
// existing executable graph is updated in place when the topology allows).
int capture_step(cr_handle *h, int precision) {
    Krylov &K = h->kry;
    const int slot = precision == CR_FP64 ? 0 : 1;
    if (K.exec[slot] && K.exec_gen[slot] == h->geo_gen && K.exec_corr[slot] == h->corr.active) return CR_OK;
    CR_TRY(realspace_prepare(h, precision));  // allocations and one-off work stay outside the graph
    if (h->corr.active) CR_TRY(correction_prepare(h));
    const long long l0 = h->launches, f0 = h->fft_execs;
    CR_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int st = record_step(h, precision);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    K.exec_kernels[slot] = h->launches - l0;
    K.exec_ffts[slot] = h->fft_execs - f0;
    h->launches = l0;  // nothing ran yet
    h->fft_execs = f0;
    if (st != CR_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return st != CR_OK ? st : fail(h, CR_CUDA_ERROR, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    if (K.exec[slot]) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(K.exec[slot], graph, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(K.exec[slot]);
            K.exec[slot] = nullptr;
        }
    }
    if (!K.exec[slot]) {
        const cudaError_t ei = cudaGraphInstantiate(&K.exec[slot], graph, 0);
        if (ei != cudaSuccess) {
            K.exec[slot] = nullptr;
            cudaGraphDestroy(graph);
            cudaGetLastError();
            return fail(h, CR_CUDA_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        }
    }
    cudaGraphDestroy(graph);
    K.exec_gen[slot] = h->geo_gen;
    K.exec_corr[slot] = h->corr.active;
    return CR_OK;
}

// One Arnoldi cycle by graph launches: at most min(m, budget) steps, stopping where the
// host loop would.  On return H and g hold the cycle's rotated Hessenberg and
// right-hand side, *cols the columns completed.
int cycle_graph(cr_handle *h, int precision, double beta, double atol, int budget, OpCount &oc, int *cols,
                std::vector<double> &H, std::vector<double> &g) {
    Krylov &K = h->kry;
    const int m = K.m;
    const int slot = precision == CR_FP64 ? 0 : 1;
    CR_TRY(capture_step(h, precision));
    init_cycle_kernel<<<blocks_for(m + 1, 128), 128, 0, h->stream>>>(m, beta, atol,
                                                                     reinterpret_cast<ArnoldiState *>(K.state), K.g);
    CR_LAUNCH(h, "init_cycle_kernel");
    const ArnoldiState *hs = reinterpret_cast<const ArnoldiState *>(K.h_state);
    int launched = 0;
    while (launched < m && launched < budget) {
        CR_CUDA(h, cudaGraphLaunch(K.exec[slot], h->stream));
        ++launched;
        ++h->graph_launches;
        h->launches += K.exec_kernels[slot];
        h->fft_execs += K.exec_ffts[slot];
        if (precision == CR_FP64) ++oc.fp64;
        else ++oc.fp32;
        CR_CUDA(h, cudaStreamSynchronize(h->stream));
        if (hs->frozen) break;
    }
    if (hs->stop == 2) return fail(h, CR_NUMERICAL, "non-finite Arnoldi norm");
    const int j = hs->j;
    CR_CUDA(h, cudaMemcpyAsync(K.h_hg, K.H, (size_t)(m + 1) * m * sizeof(double), cudaMemcpyDeviceToHost,
                               h->stream));
    CR_CUDA(h, cudaMemcpyAsync(K.h_hg + (size_t)(m + 1) * m, K.g, (m + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                               h->stream));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    std::copy(K.h_hg, K.h_hg + (size_t)(m + 1) * m, H.begin());
    std::copy(K.h_hg + (size_t)(m + 1) * m, K.h_hg + (size_t)(m + 1) * m + (m + 1), g.begin());
    *cols = j;
    return CR_OK;
}

// Restarted right-preconditioned FGMRES(m) on A_prec x = b with absolute tolerance
// `atol` on ||b - A_prec x||.  x holds the initial guess.  Returns CR_OK or
// CR_NOT_CONVERGED; *iters accumulates iterations, *restarts restart cycles.
enum { kResidualCompute = 0, kResidualIsB = 1, kResidualReady = 2 };

int fgmres(cr_handle *h, int precision, double *x, const double *b, int r_mode, double atol, int maxit,
           int *iters, int *restarts, double *final_norm, OpCount &oc, bool single_cycle = false) {
    Krylov &K = h->kry;
    const int n = K.n, m = K.m;
    const int nb = vec_blocks(n);
    double *r = K.r;
    if (r_mode == kResidualIsB) {
        CR_CUDA(h, cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    } else if (r_mode == kResidualCompute) {
        CR_TRY(op_apply(h, precision, x, r, oc));
        residual_kernel<<<nb, 256, 0, h->stream>>>(n, b, r);
        CR_LAUNCH(h, "residual_kernel");
    }
    double beta = 0;
    CR_TRY(norm(h, r, &beta));
    if (!std::isfinite(beta)) return fail(h, CR_NUMERICAL, "non-finite residual");
    std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1), y(m);
    int it = 0;
    while (beta > atol && it < maxit) {
        scale_kernel<<<nb, 256, 0, h->stream>>>(n, 1.0 / beta, r, K.V);
        CR_LAUNCH(h, "scale_kernel");
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        bool stop = false;
        if (graph_mode(h)) {
            CR_TRY(cycle_graph(h, precision, beta, atol, maxit - it, oc, &j, H, g));
            it += j;
            stop = true;  // the eager loop below is skipped
        }
        for (; j < m && it < maxit && !stop; ++j) {
            double *vj = K.V + (size_t)j * n;
            double *zj = K.Z + (size_t)j * n;
            CR_TRY(precondition_step(h, vj, zj));
            CR_TRY(op_apply(h, precision, zj, K.w, oc));
            // classical Gram-Schmidt, twice
            CR_TRY(dots(h, j + 1, K.V, K.w, K.hcol));
            project_kernel<<<nb, 256, 0, h->stream>>>(n, j + 1, K.V, K.hcol, K.w);
            CR_LAUNCH(h, "project_kernel");
            CR_TRY(dots(h, j + 1, K.V, K.w, K.hcol + (m + 1)));
            project_kernel<<<nb, 256, 0, h->stream>>>(n, j + 1, K.V, K.hcol + (m + 1), K.w);
            CR_LAUNCH(h, "project_kernel");
            CR_TRY(dots(h, 1, K.w, K.w, K.hcol + 2 * (m + 1)));
            CR_CUDA(h, cudaMemcpyAsync(K.h_pinned, K.hcol, 3 * (m + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                                       h->stream));
            CR_CUDA(h, cudaStreamSynchronize(h->stream));
            const double *h1 = K.h_pinned, *h2 = K.h_pinned + (m + 1);
            const double hn = std::sqrt(std::max(0.0, K.h_pinned[2 * (m + 1)]));
            if (!std::isfinite(hn)) return fail(h, CR_NUMERICAL, "non-finite Arnoldi norm");
            for (int k = 0; k <= j; ++k) H[(size_t)k * m + j] = h1[k] + h2[k];
            H[(size_t)(j + 1) * m + j] = hn;
            if (hn > 0) {
                scale_kernel<<<nb, 256, 0, h->stream>>>(n, 1.0 / hn, K.w, K.V + (size_t)(j + 1) * n);
                CR_LAUNCH(h, "scale_kernel");
            }
            for (int k = 0; k < j; ++k) {
                const double a = H[(size_t)k * m + j], c = H[(size_t)(k + 1) * m + j];
                H[(size_t)k * m + j] = cs[k] * a + sn[k] * c;
                H[(size_t)(k + 1) * m + j] = -sn[k] * a + cs[k] * c;
            }
            const double a = H[(size_t)j * m + j], c = H[(size_t)(j + 1) * m + j];
            const double den = std::hypot(a, c);
            cs[j] = den > 0 ? a / den : 1.0;
            sn[j] = den > 0 ? c / den : 0.0;
            H[(size_t)j * m + j] = den;
            H[(size_t)(j + 1) * m + j] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++it;
            if (std::fabs(g[j + 1]) <= atol || hn == 0.0) stop = true;
        }
        // y = H^{-1} g (upper triangular j x j), x += Z y
        for (int rr = j - 1; rr >= 0; --rr) {
            double acc = g[rr];
            for (int k = rr + 1; k < j; ++k) acc -= H[(size_t)rr * m + k] * y[k];
            y[rr] = H[(size_t)rr * m + rr] != 0.0 ? acc / H[(size_t)rr * m + rr] : 0.0;
        }
        CR_CUDA(h, cudaMemcpyAsync(K.yvec, y.data(), j * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        update_kernel<<<nb, 256, 0, h->stream>>>(n, j, K.Z, K.yvec, x);
        CR_LAUNCH(h, "update_kernel");
        K.last_cols = j;
        ++*restarts;
        if (single_cycle) {
            // the caller recomputes the residual in higher precision
            beta = std::fabs(g[j]);
            break;
        }
        // true residual of this operator
        CR_TRY(op_apply(h, precision, x, r, oc));
        residual_kernel<<<nb, 256, 0, h->stream>>>(n, b, r);
        CR_LAUNCH(h, "residual_kernel");
        CR_TRY(norm(h, r, &beta));
        if (!std::isfinite(beta)) return fail(h, CR_NUMERICAL, "non-finite residual");
    }
    *iters += it;
    *final_norm = beta;
    return beta <= atol ? CR_OK : CR_NOT_CONVERGED;
}

// Learned start: x += sum_j c_j D_j with c minimising ||r - sum_j c_j A D_j|| over the
// caller's guess directions D (h->d_guess, k of them), then the potential refit; r is
// recomputed with the FP64 operator.  The k x k normal equations are solved in FP64 on
// the host (Gaussian elimination with partial pivoting on a slightly shifted Gram matrix;
// a direction whose pivot vanishes gets weight 0).
int learned_start(cr_handle *h, int precision, double *x, const double *b, OpCount &oc, double *rnorm) {
    Krylov &K = h->kry;
    const int n = K.n, nb = vec_blocks(n);
    const int k = std::min(h->n_guess, K.m + 1);
    if (k > 0) {
        double *W = K.V;  // A D_j in the basis storage (free before the solve)
        for (int j = 0; j < k; ++j) CR_TRY(op_apply(h, precision, h->d_guess + (size_t)j * n, W + (size_t)j * n, oc));
        std::vector<double> G((size_t)k * k), rhs(k);
        for (int l = 0; l < k; ++l) {
            CR_TRY(dots(h, k, W, W + (size_t)l * n, K.hcol));
            CR_CUDA(h, cudaMemcpyAsync(K.h_pinned, K.hcol, k * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CR_CUDA(h, cudaStreamSynchronize(h->stream));
            for (int j = 0; j < k; ++j) G[(size_t)j * k + l] = K.h_pinned[j];
        }
        CR_TRY(dots(h, k, W, K.r, K.hcol));
        CR_CUDA(h, cudaMemcpyAsync(K.h_pinned, K.hcol, k * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CR_CUDA(h, cudaStreamSynchronize(h->stream));
        for (int j = 0; j < k; ++j) rhs[j] = K.h_pinned[j];
        double tr = 0;
        for (int j = 0; j < k; ++j) tr += G[(size_t)j * k + j];
        for (int j = 0; j < k; ++j) G[(size_t)j * k + j] += 1e-13 * tr + 1e-300;
        std::vector<int> piv(k);
        std::vector<double> c(k, 0.0);
        std::vector<bool> dead(k, false);
        for (int j = 0; j < k; ++j) piv[j] = j;
        for (int col = 0; col < k; ++col) {
            int best = col;
            for (int r = col + 1; r < k; ++r)
                if (std::fabs(G[(size_t)r * k + col]) > std::fabs(G[(size_t)best * k + col])) best = r;
            if (!(std::fabs(G[(size_t)best * k + col]) > 1e-14 * tr)) {
                dead[col] = true;
                continue;
            }
            if (best != col) {
                for (int q = 0; q < k; ++q) std::swap(G[(size_t)best * k + q], G[(size_t)col * k + q]);
                std::swap(rhs[best], rhs[col]);
            }
            for (int r = col + 1; r < k; ++r) {
                const double f = G[(size_t)r * k + col] / G[(size_t)col * k + col];
                for (int q = col; q < k; ++q) G[(size_t)r * k + q] -= f * G[(size_t)col * k + q];
                rhs[r] -= f * rhs[col];
            }
        }
        for (int r = k - 1; r >= 0; --r) {
            if (dead[r]) continue;
            double acc = rhs[r];
            for (int q = r + 1; q < k; ++q) acc -= G[(size_t)r * k + q] * c[q];
            c[r] = acc / G[(size_t)r * k + r];
            if (!std::isfinite(c[r])) c[r] = 0.0;
        }
        for (int j = 0; j < k; ++j)
            if (c[j] != 0.0) {
                axpy_kernel<<<nb, 256, 0, h->stream>>>(n, c[j], h->d_guess + (size_t)j * n, x);
                CR_LAUNCH(h, "axpy_kernel");
            }
        CR_TRY(op_apply(h, CR_FP64, x, K.r, oc));
        residual_kernel<<<nb, 256, 0, h->stream>>>(n, b, K.r);
        CR_LAUNCH(h, "residual_kernel");
    }
    if (h->B > 0) {
        phi_refit_kernel<<<blocks_for((long)h->B * 32, 256), 256, 0, h->stream>>>(h->N, h->B, h->d_body_start,
                                                                                 h->d_body_members, x, K.r);
        CR_LAUNCH(h, "phi_refit_kernel");
    }
    CR_TRY(norm(h, K.r, rnorm));
    if (!std::isfinite(*rnorm)) return fail(h, CR_NUMERICAL, "non-finite residual");
    return CR_OK;
}

}  // namespace

int krylov_alloc(cr_handle *h) {
    Krylov &K = h->kry;
    krylov_free(h);
    K.n = h->N + h->B;
    K.m = h->user.restart > 0 ? h->user.restart : 10;
    K.nblocks = vec_blocks(K.n);
    const size_t n = (size_t)K.n, m = (size_t)K.m;
    CR_TRY(dalloc(h, &K.V, (m + 1) * n));
    CR_TRY(dalloc(h, &K.Z, m * n));
    CR_TRY(dalloc(h, &K.w, n));
    CR_TRY(dalloc(h, &K.r, n));
    CR_TRY(dalloc(h, &K.b, n));
    CR_TRY(dalloc(h, &K.x, n));
    CR_TRY(dalloc(h, &K.d, n));
    CR_TRY(dalloc(h, &K.rr, n));
    CR_TRY(dalloc(h, &K.partial, (size_t)K.nblocks * (m + 2)));
    CR_TRY(dalloc(h, &K.hcol, 3 * (m + 1)));
    CR_TRY(dalloc(h, &K.yvec, m));
    CR_CUDA(h, cudaMallocHost((void **)&K.h_pinned, 3 * (m + 1) * sizeof(double)));
    CR_TRY(dalloc(h, &K.H, (m + 1) * m));
    CR_TRY(dalloc(h, &K.cs, m));
    CR_TRY(dalloc(h, &K.sn, m));
    CR_TRY(dalloc(h, &K.g, m + 1));
    CR_TRY(dalloc(h, &K.sin, n));
    CR_TRY(dalloc(h, &K.sz, n));
    CR_TRY(dalloc(h, &K.state, (sizeof(ArnoldiState) + sizeof(int) - 1) / sizeof(int)));
    CR_CUDA(h, cudaMallocHost(&K.h_state, sizeof(ArnoldiState)));
    CR_CUDA(h, cudaMallocHost((void **)&K.h_hg, ((m + 1) * m + (m + 1)) * sizeof(double)));
    std::memset(K.h_state, 0, sizeof(ArnoldiState));
    return CR_OK;
}

void krylov_free(cr_handle *h) {
    Krylov &K = h->kry;
    dfree(&K.V);
    dfree(&K.Z);
    dfree(&K.w);
    dfree(&K.r);
    dfree(&K.b);
    dfree(&K.x);
    dfree(&K.d);
    dfree(&K.rr);
    dfree(&K.partial);
    dfree(&K.hcol);
    dfree(&K.yvec);
    if (K.h_pinned) cudaFreeHost(K.h_pinned);
    K.h_pinned = nullptr;
    dfree(&K.H);
    dfree(&K.cs);
    dfree(&K.sn);
    dfree(&K.g);
    dfree(&K.sin);
    dfree(&K.sz);
    dfree(&K.state);
    if (K.h_state) cudaFreeHost(K.h_state);
    if (K.h_hg) cudaFreeHost(K.h_hg);
    K.h_state = nullptr;
    K.h_hg = nullptr;
    for (int s = 0; s < 2; ++s) {
        if (K.exec[s]) cudaGraphExecDestroy(K.exec[s]);
        K.exec[s] = nullptr;
        K.exec_gen[s] = -1;
    }
}

// The coarse level of the two-level preconditioner for this geometry, built on the
// handle's high-priority side stream while the stored real-space values of the geometry
// are built on the main stream: the Gauss-Jordan sweep keeps few multiprocessors busy and
// the values pass fills the rest.  The values are queued first, before the coarse set-up's
// host waits (which then wait on the side stream only).
static int prepare_overlapped(cr_handle *h) {
    const bool build = h->user.precond == CR_PRECOND_TWO_LEVEL && h->coarse.gen != h->geo_gen;
    if (!build || !h->side || h->prof.on) return coarse_prepare(h);
    cudaStream_t main = h->stream;
    CR_CUDA(h, cudaEventRecord(h->ev_fork, main));
    CR_CUDA(h, cudaStreamWaitEvent(h->side, h->ev_fork, 0));
    CR_TRY(realspace_prepare(h, h->user.precision == CR_FP64 ? CR_FP64 : CR_FP32));
    h->stream = h->side;
    int st = coarse_prepare(h);
    if (st == CR_OK) st = check_cuda(h, cudaEventRecord(h->ev_join, h->side), "cudaEventRecord");
    h->stream = main;
    CR_CUDA(h, cudaStreamWaitEvent(main, h->ev_join, 0));
    return st;
}

int solve(cr_handle *h, double *x, const double *b, cr_solve_stats *st) {
    Krylov &K = h->kry;
    const int n = K.n;
    const int nb = vec_blocks(n);
    const double tol = h->user.gmres_tol > 0 ? h->user.gmres_tol : h->user.errortol;
    const int maxit = h->user.maxiter > 0 ? h->user.maxiter : 100;
    cr_solve_stats s{};
    OpCount oc;
    double bnorm = 0, rnorm = 0;
    CR_TRY(prepare_overlapped(h));  // two-level preconditioner: coarse level of this geometry
    CR_TRY(norm(h, b, &bnorm));
    if (!std::isfinite(bnorm)) return fail(h, CR_NUMERICAL, "non-finite right-hand side");
    const double atol = tol * bnorm;
    // initial FP64 residual r0 = b - A x0; from a zero start A x0 is exactly zero (no
    // charge reaches the mesh or a pair sum), so r0 = b without an operator application
    double xnorm = 0;
    CR_TRY(norm(h, x, &xnorm));
    if (xnorm == 0.0) {
        CR_CUDA(h, cudaMemcpyAsync(K.r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    } else {
        CR_TRY(op_apply(h, CR_FP64, x, K.r, oc));
        residual_kernel<<<nb, 256, 0, h->stream>>>(n, b, K.r);
        CR_LAUNCH(h, "residual_kernel");
    }
    CR_TRY(norm(h, K.r, &rnorm));
    if (!std::isfinite(rnorm)) return fail(h, CR_NUMERICAL, "non-finite residual");
    s.initial_residual = bnorm > 0 ? rnorm / bnorm : rnorm;
    const bool learned = h->user.learned != 0;
    if (learned) {
        CR_TRY(learned_start(h, h->user.precision == CR_FP64 ? CR_FP64 : CR_FP32, x, b, oc, &rnorm));
        s.learned_residual = bnorm > 0 ? rnorm / bnorm : rnorm;
        // the guess counts as used when it lowered the initial residual
        s.used_learned_guess = s.learned_residual < 0.999 * s.initial_residual ? 1 : 0;
    }
    // learned correction of the preconditioner: used in this solve only if it reduces the
    // initial residual more than the plain preconditioner in one step
    h->corr.active = 0;
    if (h->corr.net) {
        CR_TRY(correction_decide(h, h->user.precision == CR_FP64 ? CR_FP64 : CR_FP32, K.r, K.w));
        s.used_learned_correction = h->corr.active;
        s.correction_reduction[0] = h->corr.last_rho[0];
        s.correction_reduction[1] = h->corr.last_rho[1];
    }
    int status = CR_OK;
    if (h->user.precision != CR_MIXED) {
        status = fgmres(h, h->user.precision == CR_FP32 ? CR_FP32 : CR_FP64, x, b, kResidualReady, atol, maxit,
                        &s.iterations, &s.restarts, &rnorm, oc);
        if (status != CR_OK && status != CR_NOT_CONVERGED) return status;
    } else {
        // FP64 iterative refinement around FP32 inner solves: K.rr = b - A64 x,
        // solve A32 d ~= K.rr from d = 0, x += d.
        CR_CUDA(h, cudaMemcpyAsync(K.rr, K.r, n * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        for (int outer = 0; outer < 20; ++outer) {
            if (rnorm <= atol || s.iterations >= maxit) break;
            ++s.refinements;
            // one inner cycle (up to `restart` FP32 iterations): three decades while the
            // target is more than four decades away, then to 0.3 of the target.  The FP32
            // operator's rounding is relative to the vector it multiplies, so a correction
            // solved a few decades stays far above it, while one FP32 solve carried from
            // the full right-hand side to 1e-6 slows where that rounding reaches the
            // residual (162k charges: 55 -> 46 iterations)
            const double want = 0.3 * atol / rnorm;
            const double inner_rel = std::min(0.5, want >= 1e-4 ? want : 1e-3);
            CR_CUDA(h, cudaMemsetAsync(K.d, 0, n * sizeof(double), h->stream));
            double inner_norm = 0;
            int ist = fgmres(h, CR_FP32, K.d, K.rr, kResidualIsB, inner_rel * rnorm, maxit - s.iterations,
                             &s.iterations, &s.restarts, &inner_norm, oc, true);
            if (ist != CR_OK && ist != CR_NOT_CONVERGED) return ist;
            axpy_kernel<<<nb, 256, 0, h->stream>>>(n, 1.0, K.d, x);
            CR_LAUNCH(h, "axpy_kernel");
            CR_TRY(op_apply(h, CR_FP64, x, K.rr, oc));
            residual_kernel<<<nb, 256, 0, h->stream>>>(n, b, K.rr);
            CR_LAUNCH(h, "residual_kernel");
            CR_TRY(norm(h, K.rr, &rnorm));
            if (!std::isfinite(rnorm)) return fail(h, CR_NUMERICAL, "non-finite residual");
        }
        status = rnorm <= atol ? CR_OK : CR_NOT_CONVERGED;
    }
    if (h->user.precision == CR_FP32) {
        // the FP32 loop judged its own operator; report the FP64 residual
        CR_TRY(op_apply(h, CR_FP64, x, K.w, oc));
        residual_kernel<<<nb, 256, 0, h->stream>>>(n, b, K.w);
        CR_LAUNCH(h, "residual_kernel");
        CR_TRY(norm(h, K.w, &rnorm));
    }
    s.final_residual = bnorm > 0 ? rnorm / bnorm : rnorm;
    h->n_guess = 0;  // directions apply to one solve
    s.converged = rnorm <= atol ? 1 : 0;
    s.matvecs_fp64 = oc.fp64;
    s.matvecs_fp32 = oc.fp32;
    if (st) {
        const double ms = st->solve_ms;
        *st = s;
        st->solve_ms = ms;
    }
    return s.converged ? CR_OK : (status == CR_OK ? CR_NOT_CONVERGED : status);
}

}  // namespace cr
