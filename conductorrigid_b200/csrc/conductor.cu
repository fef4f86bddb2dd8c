// conductor.cu -- the conductor-response preconditioner.
//
// The reference preconditions with a diagonal scaling (ConductorRigid.cu:816-859).
// This alternative inverts, for every body, its own block of the saddle-point system
// with the free-space mutual potential of unit shells,
//
//   A_b = [ -K_b  1 ]    K_b[k][l] = (4 - d)/(16 pi)   d < 2   (overlapping shells)
//         [ 1^T   0 ]              = 1/(4 pi d)        d >= 2
//                                  = 1/(4 pi)          k == l  (self)
//
// i.e. the exact response of the isolated conductor.  With u = K^-1 1 and s = 1^T u,
// z = A_b^-1 [r_q; r_phi] is  Phi = (r_phi + u.r_q)/s,  q = Phi u - K^-1 r_q.
// Rigid motion keeps every intra-body distance, so the block of a body never changes
// and bodies with the same shape share one inverse: shapes are grouped on the host
// (distance matrices compared entry by entry), factorised once in FP64 (Cholesky),
// and applied on the device, one CTA per body.  In flexible GMRES any fixed or varying
// preconditioner leaves the solution unchanged; only the iteration count moves.
#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>
#include <vector>

#include "cr_internal.cuh"

namespace cr {

namespace {

double shell_kernel(double d) {
    if (d == 0.0) return 1.0 / (4.0 * kPi);
    return d < 2.0 ? (4.0 - d) / (16.0 * kPi) : 1.0 / (4.0 * kPi * d);
}

// In-place Cholesky K = L L^T (lower, row-major n x n); false if not positive definite.
bool cholesky(std::vector<double> &a, int n) {
    for (int j = 0; j < n; ++j) {
        double d = a[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= a[(size_t)j * n + k] * a[(size_t)j * n + k];
        if (!(d > 0.0)) return false;
        d = std::sqrt(d);
        a[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double v = a[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) v -= a[(size_t)i * n + k] * a[(size_t)j * n + k];
            a[(size_t)i * n + j] = v / d;
        }
    }
    return true;
}

// x = (L L^T)^-1 b in place
void chol_solve(const std::vector<double> &l, int n, double *x) {
    for (int i = 0; i < n; ++i) {
        double v = x[i];
        for (int k = 0; k < i; ++k) v -= l[(size_t)i * n + k] * x[k];
        x[i] = v / l[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double v = x[i];
        for (int k = i + 1; k < n; ++k) v -= l[(size_t)k * n + i] * x[k];
        x[i] = v / l[(size_t)i * n + i];
    }
}

// (body b: the body of conductor_apply_kernel and of its lockstep-batch form)
__device__ __forceinline__ void conductor_apply_body(int b, int N, const int *__restrict__ body_start,
                                                     const int *__restrict__ members,
                                                     const int *__restrict__ body_shape,
                                                     const int *__restrict__ shape_n,
                                                     const long long *__restrict__ shape_mat,
                                                     const int *__restrict__ shape_vec,
                                                     const double *__restrict__ kinv,
                                                     const double *__restrict__ uvec,
                                                     const double *__restrict__ inv_s, const double *__restrict__ v,
                                                     double *__restrict__ z) {
    extern __shared__ double sh[];
    __shared__ double red[32];
    const int s = body_shape[b];
    const int n = shape_n[s];
    const int beg = body_start[b];
    const double *K = kinv + shape_mat[s];
    const double *u = uvec + shape_vec[s];
    double *r = sh;
    double part = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const double rk = v[members[beg + k]];
        r[k] = rk;
        part += u[k] * rk;
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const double phi = (v[N + b] + red[0]) * inv_s[s];
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < n; ++j) acc += K[(size_t)j * n + k] * r[j];  // column-major
        z[members[beg + k]] = phi * u[k] - acc;
    }
    if (threadIdx.x == 0) z[N + b] = phi;
}

__global__ void conductor_apply_kernel(int N, int B, const int *__restrict__ body_start,
                                       const int *__restrict__ members, const int *__restrict__ body_shape,
                                       const int *__restrict__ shape_n, const long long *__restrict__ shape_mat,
                                       const int *__restrict__ shape_vec, const double *__restrict__ kinv,
                                       const double *__restrict__ uvec, const double *__restrict__ inv_s,
                                       const double *__restrict__ v, double *__restrict__ z) {
    if ((int)blockIdx.x >= B) return;
    conductor_apply_body(blockIdx.x, N, body_start, members, body_shape, shape_n, shape_mat, shape_vec, kinv, uvec,
                         inv_s, v, z);
}

// lockstep batch: one CTA per (replica, body); the input is the coarse level's t for
// replicas whose coarse level is active when from_coarse is set
__global__ void conductor_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                       const int *__restrict__ mask, int xin, int from_coarse, int zout) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &r = reps[it.x];
    const double *v = from_coarse && r.coarse ? r.ct : r.vec[xin];
    conductor_apply_body(it.y, r.N, r.body_start, r.body_members, r.body_shape, r.shape_n, r.shape_mat, r.shape_vec,
                         r.kinv, r.uvec, r.inv_s, v, r.vec[zout]);
}

}  // namespace

int batch_conductor(cr_batch *bt, const int *mask, int xin, bool from_coarse, int zout, cudaStream_t s) {
    if (bt->n_items[BL_BODIES] == 0) return CR_OK;
    conductor_batch_kernel<<<bt->n_items[BL_BODIES], bt->cond_threads, bt->cond_smem, s>>>(
        bt->d_reps, bt->d_items[BL_BODIES], mask, xin, from_coarse ? 1 : 0, zout);
    ++bt->launches;
    return batch_check(bt, cudaGetLastError(), "conductor_batch_kernel");
}

void conductor_free(cr_handle *h) {
    dfree(&h->cond.d_body_shape);
    dfree(&h->cond.d_shape_n);
    dfree(&h->cond.d_shape_mat);
    dfree(&h->cond.d_shape_vec);
    dfree(&h->cond.d_kinv);
    dfree(&h->cond.d_u);
    dfree(&h->cond.d_invs);
    h->cond.ready = false;
    h->cond.n_shapes = 0;
}

// Group bodies by shape and factorise each shape (positions from the current geometry).
int conductor_setup(cr_handle *h) {
    const int N = h->N, B = h->B;
    ConductorPrecond &C = h->cond;
    conductor_free(h);
    if (B == 0) {
        C.ready = true;
        return CR_OK;
    }
    std::vector<double4> pos(N);
    CR_CUDA(h, cudaMemcpyAsync(pos.data(), h->m64.pos, N * sizeof(double4), cudaMemcpyDeviceToHost, h->stream));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    const std::vector<int> &start = h->h_body_start;
    const std::vector<int> &mem = h->h_body_members;
    int max_n = 0;
    for (int b = 0; b < B; ++b) max_n = std::max(max_n, start[b + 1] - start[b]);
    if (max_n > 4096) return fail(h, CR_BAD_PARAM, "conductor preconditioner: a body holds more than 4096 beads");
    auto rel = [&](int b, int k, double *r) {
        const double4 a = pos[mem[start[b]]], c = pos[mem[start[b] + k]];
        const double d[3] = {c.x - a.x, c.y - a.y, c.z - a.z};
        for (int e = 0; e < 3; ++e) r[e] = d[e] - h->L[e] * std::rint(d[e] / h->L[e]);
    };
    auto dist2 = [&](int b, int k, int l) {
        double rk[3], rl[3];
        rel(b, k, rk);
        rel(b, l, rl);
        const double dx = rk[0] - rl[0], dy = rk[1] - rl[1], dz = rk[2] - rl[2];
        return dx * dx + dy * dy + dz * dz;
    };
    // shape signatures: (n, sum d^2, sum d^4) bucketed, confirmed entry by entry
    std::map<std::tuple<int, long long, long long>, std::vector<int>> buckets;
    std::vector<int> body_shape(B, -1), reps;
    for (int b = 0; b < B; ++b) {
        const int n = start[b + 1] - start[b];
        double s2 = 0, s4 = 0;
        for (int k = 0; k < n; ++k)
            for (int l = k + 1; l < n; ++l) {
                const double d2 = dist2(b, k, l);
                s2 += d2;
                s4 += d2 * d2;
            }
        auto key = std::make_tuple(n, std::llround(s2 * 1e4), std::llround(s4 * 1e2));
        auto &cand = buckets[key];
        int found = -1;
        for (int sidx : cand) {
            const int rb = reps[sidx];
            bool same = true;
            for (int k = 0; k < n && same; ++k)
                for (int l = k + 1; l < n; ++l)
                    if (std::fabs(dist2(b, k, l) - dist2(rb, k, l)) > 1e-9 * (1.0 + dist2(rb, k, l))) {
                        same = false;
                        break;
                    }
            if (same) {
                found = sidx;
                break;
            }
        }
        if (found < 0) {
            found = (int)reps.size();
            reps.push_back(b);
            cand.push_back(found);
        }
        body_shape[b] = found;
    }
    const int S = (int)reps.size();
    std::vector<int> shape_n(S), shape_vec(S);
    std::vector<long long> shape_mat(S);
    long long mat_total = 0;
    int vec_total = 0;
    for (int s = 0; s < S; ++s) {
        shape_n[s] = start[reps[s] + 1] - start[reps[s]];
        shape_mat[s] = mat_total;
        shape_vec[s] = vec_total;
        mat_total += (long long)shape_n[s] * shape_n[s];
        vec_total += shape_n[s];
    }
    std::vector<double> kinv((size_t)mat_total), u((size_t)vec_total), invs(S);
    for (int s = 0; s < S; ++s) {
        const int n = shape_n[s], rb = reps[s];
        std::vector<double> K((size_t)n * n);
        for (int k = 0; k < n; ++k)
            for (int l = 0; l < n; ++l) K[(size_t)k * n + l] = shell_kernel(k == l ? 0.0 : std::sqrt(dist2(rb, k, l)));
        if (!cholesky(K, n))
            return fail(h, CR_NUMERICAL, "conductor preconditioner: a body's shell matrix is not positive definite");
        std::vector<double> col(n);
        for (int j = 0; j < n; ++j) {  // column j of K^-1, stored column-major
            std::fill(col.begin(), col.end(), 0.0);
            col[j] = 1.0;
            chol_solve(K, n, col.data());
            for (int k = 0; k < n; ++k) kinv[(size_t)shape_mat[s] + (size_t)j * n + k] = col[k];
        }
        std::fill(col.begin(), col.end(), 1.0);
        chol_solve(K, n, col.data());
        double ss = 0.0;
        for (int k = 0; k < n; ++k) {
            u[(size_t)shape_vec[s] + k] = col[k];
            ss += col[k];
        }
        invs[s] = 1.0 / ss;
    }
    CR_TRY(dalloc(h, &C.d_body_shape, (size_t)B));
    CR_TRY(dalloc(h, &C.d_shape_n, (size_t)S));
    CR_TRY(dalloc(h, &C.d_shape_mat, (size_t)S));
    CR_TRY(dalloc(h, &C.d_shape_vec, (size_t)S));
    CR_TRY(dalloc(h, &C.d_kinv, (size_t)mat_total));
    CR_TRY(dalloc(h, &C.d_u, (size_t)vec_total));
    CR_TRY(dalloc(h, &C.d_invs, (size_t)S));
    CR_CUDA(h, cudaMemcpy(C.d_body_shape, body_shape.data(), B * sizeof(int), cudaMemcpyHostToDevice));
    CR_CUDA(h, cudaMemcpy(C.d_shape_n, shape_n.data(), S * sizeof(int), cudaMemcpyHostToDevice));
    CR_CUDA(h, cudaMemcpy(C.d_shape_mat, shape_mat.data(), S * sizeof(long long), cudaMemcpyHostToDevice));
    CR_CUDA(h, cudaMemcpy(C.d_shape_vec, shape_vec.data(), S * sizeof(int), cudaMemcpyHostToDevice));
    CR_CUDA(h, cudaMemcpy(C.d_kinv, kinv.data(), mat_total * sizeof(double), cudaMemcpyHostToDevice));
    CR_CUDA(h, cudaMemcpy(C.d_u, u.data(), vec_total * sizeof(double), cudaMemcpyHostToDevice));
    CR_CUDA(h, cudaMemcpy(C.d_invs, invs.data(), S * sizeof(double), cudaMemcpyHostToDevice));
    C.n_shapes = S;
    C.max_n = max_n;
    C.ready = true;
    return CR_OK;
}

int conductor_apply(cr_handle *h, const double *x, double *y) {
    const ConductorPrecond &C = h->cond;
    if (!C.ready) return fail(h, CR_NOT_READY, "conductor preconditioner not set up");
    if (h->B == 0) return CR_OK;
    const size_t smem = (size_t)C.max_n * sizeof(double);
    const int threads = std::min(256, std::max(64, (C.max_n + 31) / 32 * 32));  // one pass over a body's rows
    conductor_apply_kernel<<<h->B, threads, smem, h->stream>>>(h->N, h->B, h->d_body_start, h->d_body_members,
                                                           C.d_body_shape, C.d_shape_n, C.d_shape_mat, C.d_shape_vec,
                                                           C.d_kinv, C.d_u, C.d_invs, x, y);
    CR_LAUNCH(h, "conductor_apply_kernel");
    return CR_OK;
}

}  // namespace cr
