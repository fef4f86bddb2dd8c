// guess.cu -- inputs and outputs of the learned initial guess for time stepping.
//
// Between two steps of a trajectory the solution changes because every body moved.
// The guess machinery turns the previous solution q' (at positions r', centres R') and
// the new positions (r, R) into:
//   * the transport term s_i = grad_s q'(r'_i) . delta_i: the previous surface charge
//     field, taken as fixed in the lab frame, sampled where the body's rotation carried
//     bead i (delta_i = bead displacement minus centre displacement, minimum image); the
//     surface gradient is the least-squares fit over the bead's nearest same-body beads;
//   * 48 per-bead features for the network (FP32, then standardised and packed to
//     BF16 rows): q'_i, s_i, E0.n_i, Q_b, and for each of the 8 nearest bodies k the
//     cosine n_i.u_k, the proximity 1/(1 + gap), the gap change since the last step,
//     their product with the cosine, and q'_i times the gap change;
//   * neutral directions: per-body means removed so that adding a direction to the
//     charges leaves every body's total charge (the constraint rows) unchanged.
#include <cuda_bf16.h>

#include "cr_internal.cuh"

namespace cr {

namespace {

constexpr int KB = CR_GUESS_BEAD_NEIGHBORS;   // 6
constexpr int KN = CR_GUESS_BODY_NEIGHBORS;   // 8
constexpr int NF = CR_MLP_FEATURES;           // 48

__device__ inline double mimg(double d, double L) { return d - L * rint(d / L); }

template <int K>
__device__ inline void topk_insert(double d2, int j, double *best, int *idx) {
    if (d2 >= best[K - 1]) return;
    int p = K - 1;
    while (p > 0 && best[p - 1] > d2) {
        best[p] = best[p - 1];
        idx[p] = idx[p - 1];
        --p;
    }
    best[p] = d2;
    idx[p] = j;
}

// KB nearest other beads of the same body (ties by lower index); missing -> self.
__global__ void bead_neighbors_kernel(int N, const uint32_t *__restrict__ body, const int *__restrict__ start,
                                      const int *__restrict__ members, const double *__restrict__ pos, double Lx,
                                      double Ly, double Lz, int *__restrict__ nbr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int b = body[i];
    double best[KB];
    int idx[KB];
    for (int k = 0; k < KB; ++k) {
        best[k] = 1e300;
        idx[k] = i;
    }
    const double px = pos[3 * (size_t)i], py = pos[3 * (size_t)i + 1], pz = pos[3 * (size_t)i + 2];
    for (int k = start[b]; k < start[b + 1]; ++k) {
        const int j = members[k];
        if (j == i) continue;
        const double dx = mimg(pos[3 * (size_t)j] - px, Lx), dy = mimg(pos[3 * (size_t)j + 1] - py, Ly),
                     dz = mimg(pos[3 * (size_t)j + 2] - pz, Lz);
        topk_insert<KB>(dx * dx + dy * dy + dz * dz, j, best, idx);
    }
    for (int k = 0; k < KB; ++k) nbr[(size_t)i * KB + k] = idx[k];
}

// KN nearest other bodies by centre distance (minimum image); missing -> self.
__global__ void body_neighbors_kernel(int B, const double *__restrict__ bpos, double Lx, double Ly, double Lz,
                                      int *__restrict__ nbr) {
    __shared__ double3 tile[256];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    double best[KN];
    int idx[KN];
    for (int k = 0; k < KN; ++k) {
        best[k] = 1e300;
        idx[k] = b;
    }
    double3 c = make_double3(0, 0, 0);
    if (b < B) c = make_double3(bpos[3 * (size_t)b], bpos[3 * (size_t)b + 1], bpos[3 * (size_t)b + 2]);
    for (int t0 = 0; t0 < B; t0 += 256) {
        const int j = t0 + threadIdx.x;
        if (j < B) tile[threadIdx.x] = make_double3(bpos[3 * (size_t)j], bpos[3 * (size_t)j + 1], bpos[3 * (size_t)j + 2]);
        __syncthreads();
        const int cnt = min(256, B - t0);
        if (b < B)
            for (int u = 0; u < cnt; ++u) {
                if (t0 + u == b) continue;
                const double dx = mimg(tile[u].x - c.x, Lx), dy = mimg(tile[u].y - c.y, Ly), dz = mimg(tile[u].z - c.z, Lz);
                topk_insert<KN>(dx * dx + dy * dy + dz * dz, t0 + u, best, idx);
            }
        __syncthreads();
    }
    if (b < B)
        for (int k = 0; k < KN; ++k) nbr[(size_t)b * KN + k] = idx[k];
}

struct FeatArgs {
    int N;
    double L[3];
    double E[3];
};

__global__ void features_kernel(FeatArgs a, const uint32_t *__restrict__ body, const double *__restrict__ Q,
                                const double *__restrict__ radius, const int *__restrict__ bead_nbr,
                                const int *__restrict__ body_nbr, const double *__restrict__ q_prev,
                                const double *__restrict__ pos_prev, const double *__restrict__ bpos_prev,
                                const double *__restrict__ pos, const double *__restrict__ bpos,
                                float *__restrict__ feat, double *__restrict__ s_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    const int b = body[i];
    const double qi = q_prev[i];
    // surface gradient of q' at bead i: (D^T D + eps I) G = D^T dq over the bead neighbours
    double A[6] = {0, 0, 0, 0, 0, 0}, rhs[3] = {0, 0, 0};
    const double p0[3] = {pos_prev[3 * (size_t)i], pos_prev[3 * (size_t)i + 1], pos_prev[3 * (size_t)i + 2]};
    for (int k = 0; k < KB; ++k) {
        const int j = bead_nbr[(size_t)i * KB + k];
        if (j == i) continue;
        double d[3];
        for (int e = 0; e < 3; ++e) d[e] = mimg(pos_prev[3 * (size_t)j + e] - p0[e], a.L[e]);
        const double dq = q_prev[j] - qi;
        A[0] += d[0] * d[0];
        A[1] += d[0] * d[1];
        A[2] += d[0] * d[2];
        A[3] += d[1] * d[1];
        A[4] += d[1] * d[2];
        A[5] += d[2] * d[2];
        for (int e = 0; e < 3; ++e) rhs[e] += d[e] * dq;
    }
    const double eps = 1e-3 * (A[0] + A[3] + A[5]) + 1e-300;
    const double a00 = A[0] + eps, a01 = A[1], a02 = A[2], a11 = A[3] + eps, a12 = A[4], a22 = A[5] + eps;
    const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22, c02 = a01 * a12 - a02 * a11;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    double G[3] = {0, 0, 0};
    if (det != 0.0) {
        const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12, c22 = a00 * a11 - a01 * a01;
        G[0] = (c00 * rhs[0] + c01 * rhs[1] + c02 * rhs[2]) / det;
        G[1] = (c01 * rhs[0] + c11 * rhs[1] + c12 * rhs[2]) / det;
        G[2] = (c02 * rhs[0] + c12 * rhs[1] + c22 * rhs[2]) / det;
    }
    double n[3], delta[3];
    double nn = 0;
    for (int e = 0; e < 3; ++e) {
        const double cb = bpos[3 * (size_t)b + e];
        n[e] = mimg(pos[3 * (size_t)i + e] - cb, a.L[e]);
        nn += n[e] * n[e];
        delta[e] = mimg((pos[3 * (size_t)i + e] - pos_prev[3 * (size_t)i + e]) -
                            (cb - bpos_prev[3 * (size_t)b + e]), a.L[e]);
    }
    nn = nn > 0 ? 1.0 / sqrt(nn) : 0.0;
    for (int e = 0; e < 3; ++e) n[e] *= nn;
    const double s = G[0] * delta[0] + G[1] * delta[1] + G[2] * delta[2];
    s_out[i] = s;
    float *f = feat + (size_t)i * NF;
    f[0] = (float)qi;
    f[1] = (float)s;
    f[2] = (float)(a.E[0] * n[0] + a.E[1] * n[1] + a.E[2] * n[2]);
    f[3] = (float)Q[b];
    double first_eu = 0, first_w = 0;
    for (int k = 0; k < KN; ++k) {
        const int j = body_nbr[(size_t)b * KN + k];
        double u[3], up[3];
        double d2 = 0, dp2 = 0;
        for (int e = 0; e < 3; ++e) {
            u[e] = mimg(bpos[3 * (size_t)j + e] - bpos[3 * (size_t)b + e], a.L[e]);
            up[e] = mimg(bpos_prev[3 * (size_t)j + e] - bpos_prev[3 * (size_t)b + e], a.L[e]);
            d2 += u[e] * u[e];
            dp2 += up[e] * up[e];
        }
        const double d = sqrt(d2), dp = sqrt(dp2);
        float *g = f + 4 + 5 * k;
        if (j == b || d == 0.0) {
            for (int e = 0; e < 5; ++e) g[e] = 0.f;
            continue;
        }
        const double c = (n[0] * u[0] + n[1] * u[1] + n[2] * u[2]) / d;
        const double gap = fmax(d - radius[b] - radius[j], 0.0);
        const double w = 1.0 / (1.0 + gap);
        const double dg = 100.0 * (d - dp);
        g[0] = (float)c;
        g[1] = (float)w;
        g[2] = (float)dg;
        g[3] = (float)(dg * w * c);
        g[4] = (float)(qi * dg);
        if (k == 0) {
            first_eu = (a.E[0] * u[0] + a.E[1] * u[1] + a.E[2] * u[2]) / d;
            first_w = w;
        }
    }
    f[44] = (float)(first_eu * first_w);
    f[45] = 0.f;
    f[46] = 0.f;
    f[47] = 0.f;
}

// sums[f] += x, sums[NF + f] += x^2 over rows (FP64)
__global__ void feature_stats_kernel(int N, const float *__restrict__ feat, double *__restrict__ sums) {
    const int f = threadIdx.x % NF;
    const int lanes = blockDim.x / NF;
    const int sub = threadIdx.x / NF;
    if (sub >= lanes) return;
    double s = 0, s2 = 0;
    for (int i = blockIdx.x * lanes + sub; i < N; i += gridDim.x * lanes) {
        const double x = feat[(size_t)i * NF + f];
        s += x;
        s2 += x * x;
    }
    atomicAdd(&sums[f], s);
    atomicAdd(&sums[NF + f], s2);
}

__global__ void feature_pack_kernel(int N, const float *__restrict__ feat, const float *__restrict__ mu,
                                    const float *__restrict__ inv_sigma, __nv_bfloat16 *__restrict__ out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)N * NF) return;
    const int f = (int)(t % NF);
    out[t] = __float2bfloat16_rn((feat[t] - mu[f]) * inv_sigma[f]);
}

__global__ void target_kernel(int N, const double *__restrict__ q, const double *__restrict__ q_prev, double inv_scale,
                              float *__restrict__ t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) t[i] = (float)((q[i] - q_prev[i]) * inv_scale);
}

// out[q rows] = scale * v - per-body mean, out[body rows] = 0   (v FP64 or FP32)
template <typename T>
__global__ void neutral_kernel(int N, int B, const int *__restrict__ start, const int *__restrict__ members,
                               const T *__restrict__ v, double scale, double *__restrict__ out) {
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= B) return;
    const int k0 = start[b], k1 = start[b + 1];
    double s = 0;
    for (int k = k0 + lane; k < k1; k += 32) s += (double)v[members[k]];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double mean = s / (double)(k1 - k0);
    for (int k = k0 + lane; k < k1; k += 32) out[members[k]] = scale * ((double)v[members[k]] - mean);
    if (lane == 0) out[N + b] = 0.0;
}

}  // namespace
}  // namespace cr

using namespace cr;

extern "C" {

int cr_bead_neighbors(cr_handle *h, const double *d_pos, int *d_nbr) {
    if (!h || !h->have_topology) return h ? fail(h, CR_NOT_READY, "topology not set") : CR_BAD_PARAM;
    if (h->N == 0) return CR_OK;
    if (!d_pos || !d_nbr) return fail(h, CR_BAD_PARAM, "null array");
    bead_neighbors_kernel<<<blocks_for(h->N, 128), 128, 0, h->stream>>>(h->N, h->d_body, h->d_body_start,
                                                                       h->d_body_members, d_pos, h->L[0], h->L[1],
                                                                       h->L[2], d_nbr);
    CR_LAUNCH(h, "bead_neighbors_kernel");
    return CR_OK;
}

int cr_body_neighbors(cr_handle *h, const double *d_body_pos, int *d_nbr) {
    if (!h || !h->have_topology) return h ? fail(h, CR_NOT_READY, "topology not set") : CR_BAD_PARAM;
    if (h->B == 0) return CR_OK;
    if (!d_body_pos || !d_nbr) return fail(h, CR_BAD_PARAM, "null array");
    body_neighbors_kernel<<<blocks_for(h->B, 256), 256, 0, h->stream>>>(h->B, d_body_pos, h->L[0], h->L[1], h->L[2],
                                                                       d_nbr);
    CR_LAUNCH(h, "body_neighbors_kernel");
    return CR_OK;
}

int cr_guess_features(cr_handle *h, const double *d_radius, const int *d_bead_nbr, const int *d_body_nbr,
                      const double *d_q_prev, const double *d_pos_prev, const double *d_body_pos_prev,
                      const double *d_pos, const double *d_body_pos, float *d_feat, double *d_transport) {
    if (!h || !h->have_topology) return h ? fail(h, CR_NOT_READY, "topology not set") : CR_BAD_PARAM;
    if (h->N == 0) return CR_OK;
    if (!d_radius || !d_bead_nbr || !d_body_nbr || !d_q_prev || !d_pos_prev || !d_body_pos_prev || !d_pos ||
        !d_body_pos || !d_feat || !d_transport)
        return fail(h, CR_BAD_PARAM, "null array");
    FeatArgs a;
    a.N = h->N;
    for (int e = 0; e < 3; ++e) {
        a.L[e] = h->L[e];
        a.E[e] = h->field[e];
    }
    features_kernel<<<blocks_for(h->N, 128), 128, 0, h->stream>>>(a, h->d_body, h->d_Q, d_radius, d_bead_nbr,
                                                                  d_body_nbr, d_q_prev, d_pos_prev, d_body_pos_prev,
                                                                  d_pos, d_body_pos, d_feat, d_transport);
    CR_LAUNCH(h, "features_kernel");
    return CR_OK;
}

int cr_feature_stats(cr_handle *h, int n, const float *d_feat, double *d_sums) {
    if (!h || n < 0 || (n > 0 && (!d_feat || !d_sums))) return CR_BAD_PARAM;
    CR_CUDA(h, cudaMemsetAsync(d_sums, 0, 2 * NF * sizeof(double), h->stream));
    if (n == 0) return CR_OK;
    const int lanes = 5;  // 5 x 48 = 240 threads
    feature_stats_kernel<<<std::min(4 * 148, blocks_for(n, lanes)), lanes * NF, 0, h->stream>>>(n, d_feat, d_sums);
    CR_LAUNCH(h, "feature_stats_kernel");
    return CR_OK;
}

int cr_feature_pack(cr_handle *h, int n, const float *d_feat, const float *d_mu, const float *d_inv_sigma,
                    uint16_t *d_x) {
    if (!h || n < 0 || (n > 0 && (!d_feat || !d_mu || !d_inv_sigma || !d_x))) return CR_BAD_PARAM;
    if (n == 0) return CR_OK;
    feature_pack_kernel<<<blocks_for((long)n * NF, 256), 256, 0, h->stream>>>(
        n, d_feat, d_mu, d_inv_sigma, reinterpret_cast<__nv_bfloat16 *>(d_x));
    CR_LAUNCH(h, "feature_pack_kernel");
    return CR_OK;
}

int cr_guess_target(cr_handle *h, const double *d_q, const double *d_q_prev, double scale, float *d_t) {
    if (!h || !(scale > 0.0)) return h ? fail(h, CR_BAD_PARAM, "scale must be > 0") : CR_BAD_PARAM;
    if (h->N == 0) return CR_OK;
    if (!d_q || !d_q_prev || !d_t) return fail(h, CR_BAD_PARAM, "null array");
    target_kernel<<<blocks_for(h->N, 256), 256, 0, h->stream>>>(h->N, d_q, d_q_prev, 1.0 / scale, d_t);
    CR_LAUNCH(h, "target_kernel");
    return CR_OK;
}

int cr_neutral_direction(cr_handle *h, const void *d_v, int v_is_fp32, double scale, double *d_dir) {
    if (!h || !h->have_topology) return h ? fail(h, CR_NOT_READY, "topology not set") : CR_BAD_PARAM;
    if (h->B == 0) return CR_OK;
    if (!d_v || !d_dir) return fail(h, CR_BAD_PARAM, "null array");
    if (v_is_fp32)
        neutral_kernel<float><<<blocks_for((long)h->B * 32, 256), 256, 0, h->stream>>>(
            h->N, h->B, h->d_body_start, h->d_body_members, static_cast<const float *>(d_v), scale, d_dir);
    else
        neutral_kernel<double><<<blocks_for((long)h->B * 32, 256), 256, 0, h->stream>>>(
            h->N, h->B, h->d_body_start, h->d_body_members, static_cast<const double *>(d_v), scale, d_dir);
    CR_LAUNCH(h, "neutral_kernel");
    return CR_OK;
}

int cr_set_guess_directions(cr_handle *h, int n_dir, const double *d_dirs) {
    CR_TRY(h ? CR_OK : CR_BAD_PARAM);
    if (!h->have_topology) return fail(h, CR_NOT_READY, "topology not set");
    if (n_dir < 0 || n_dir > CR_MAX_GUESS_DIRECTIONS) return fail(h, CR_BAD_PARAM, "too many guess directions");
    if (n_dir > 0 && !d_dirs) return fail(h, CR_BAD_PARAM, "null directions");
    const size_t n = (size_t)h->N + h->B;
    if (n_dir > 0 && !h->d_guess) CR_TRY(dalloc(h, &h->d_guess, CR_MAX_GUESS_DIRECTIONS * n));
    if (n_dir > 0)
        CR_CUDA(h, cudaMemcpyAsync(h->d_guess, d_dirs, n_dir * n * sizeof(double), cudaMemcpyDeviceToDevice,
                                   h->stream));
    h->n_guess = n_dir;
    return CR_OK;
}

}  // extern "C"
