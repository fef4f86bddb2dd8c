// body.cu -- body-level rows of the saddle-point system and the operator assembly.
//
//   [ -M   S^T ] [ q   ]   [ -(r_i - R_b).E0 ]
//   [  S    0  ] [ Phi ] = [        Q_b      ]        (ConductorRigid.cu:1046-1050)
//
// S sums the charges of each body (sum_charges, cu:667-730, for rigid bodies and
// set_charge, cu:733-761, for free beads -- the same sum over the body's members).
// The member lists are a stable device sort of beads by body tag, so they are
// ordered by bead index and identical on every run.  All body sums are FP64 in every
// precision mode.
#include <cub/cub.cuh>

#include "cr_internal.cuh"

namespace cr {

namespace {

__global__ void body_sums_kernel(int N, int B, const int *__restrict__ start, const int *__restrict__ members,
                                 const double *__restrict__ x, double *__restrict__ y) {
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= B) return;
    double s = 0.0;
    for (int k = start[b] + lane; k < start[b + 1]; k += 32) s += x[members[k]];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[N + b] = s;
}

// ConductorRigid.cu:764-813 (free beads keep the zero of zero_array, cu:1102).
__global__ void objective_kernel(int N, int B, const double4 *__restrict__ pos, const double4 *__restrict__ bpos,
                                 const uint32_t *__restrict__ body, const uint8_t *__restrict__ rigid,
                                 const double *__restrict__ Q, double Lx, double Ly, double Lz, double Ex, double Ey,
                                 double Ez, double *__restrict__ rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        const uint32_t b = body[i];
        if (!rigid[b]) {
            rhs[i] = 0.0;
            return;
        }
        const double4 p = pos[i], c = bpos[b];
        double rx = p.x - c.x, ry = p.y - c.y, rz = p.z - c.z;
        rx -= Lx * rint(rx / Lx);
        ry -= Ly * rint(ry / Ly);
        rz -= Lz * rint(rz / Lz);
        rhs[i] = -(rx * Ex + ry * Ey + rz * Ez);
    } else if (i < N + B) {
        rhs[i] = Q[i - N];
    }
}

// ConductorRigid.cu:816-859.  Rigid-body rows 1/size (the value the reference's
// second write leaves when the rigid index equals the body tag, cu:855), free-bead
// rows 1/(4 pi) (cu:837).
__global__ void precondition_kernel(int N, int B, const uint8_t *__restrict__ rigid, const int *__restrict__ bsize,
                                    const double *__restrict__ x, double *__restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        y[i] = -4.0 * kPi * x[i];
    } else if (i < N + B) {
        const int b = i - N;
        y[i] = rigid[b] ? x[i] / (double)bsize[b] : x[i] / (4.0 * kPi);
    }
}

__global__ void iota_kernel(int n, int *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}
__global__ void count_kernel(const uint32_t *__restrict__ key, int n, int *count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(count + key[i], 1);
}

}  // namespace

// Member lists of the bodies: d_body_start[B+1], d_body_members[N], d_bsize[B].
int topology_build(cr_handle *h) {
    const int N = h->N, B = h->B;
    cudaStream_t s = h->stream;
    int *iota = nullptr, *cnt = nullptr;
    uint32_t *keys_out = nullptr;
    void *tmp = nullptr;
    size_t b1 = 0, b2 = 0;
    int st = dalloc(h, &iota, (size_t)N);
    if (st == CR_OK) st = dalloc(h, &cnt, (size_t)B + 1);
    if (st == CR_OK) st = dalloc(h, &keys_out, (size_t)N);
    if (st == CR_OK) {
        cub::DeviceRadixSort::SortPairs(nullptr, b1, h->d_body, keys_out, iota, h->d_body_members, N);
        cub::DeviceScan::ExclusiveSum(nullptr, b2, cnt, h->d_body_start, B + 1);
        st = dalloc(h, reinterpret_cast<char **>(&tmp), std::max(b1, b2) + 256);
    }
    if (st == CR_OK) {
        iota_kernel<<<blocks_for(N, 256), 256, 0, s>>>(N, iota);
        cudaMemsetAsync(cnt, 0, (B + 1) * sizeof(int), s);
        count_kernel<<<blocks_for(N, 256), 256, 0, s>>>(h->d_body, N, cnt);
        size_t bytes = std::max(b1, b2) + 256;
        st = check_cuda(h, cub::DeviceScan::ExclusiveSum(tmp, bytes, cnt, h->d_body_start, B + 1, s), "scan");
        bytes = std::max(b1, b2) + 256;
        if (st == CR_OK)
            st = check_cuda(h, cub::DeviceRadixSort::SortPairs(tmp, bytes, h->d_body, keys_out, iota,
                                                               h->d_body_members, N, 0, 32, s),
                            "sort");
        if (st == CR_OK)
            st = check_cuda(h, cudaMemcpyAsync(h->d_bsize, cnt, B * sizeof(int), cudaMemcpyDeviceToDevice, s), "copy");
        if (st == CR_OK) st = check_cuda(h, cudaStreamSynchronize(s), "topology_build");
    }
    dfree(&iota);
    dfree(&cnt);
    dfree(&keys_out);
    dfree(reinterpret_cast<char **>(&tmp));
    return st;
}

int body_sums(cr_handle *h, const double *x, double *y) {
    if (h->B == 0) return CR_OK;
    ProfScope ps(h, PROF_BODY);
    body_sums_kernel<<<blocks_for((long)h->B * 32, 256), 256, 0, h->stream>>>(h->N, h->B, h->d_body_start,
                                                                               h->d_body_members, x, y);
    CR_LAUNCH(h, "body_sums_kernel");
    return CR_OK;
}

int objective(cr_handle *h, double *rhs) {
    const int n = h->N + h->B;
    objective_kernel<<<blocks_for(n, 256), 256, 0, h->stream>>>(h->N, h->B, h->m64.pos, h->d_bpos, h->d_body,
                                                                 h->d_rigid, h->d_Q, h->L[0], h->L[1], h->L[2],
                                                                 h->field[0], h->field[1], h->field[2], rhs);
    CR_LAUNCH(h, "objective_kernel");
    return CR_OK;
}

int precondition(cr_handle *h, const double *x, double *y) {
    ProfScope ps(h, PROF_PRECOND);
    if (h->user.precond == CR_PRECOND_CONDUCTOR) return conductor_apply(h, x, y);
    if (h->user.precond == CR_PRECOND_TWO_LEVEL) return coarse_apply(h, x, y);
    const int n = h->N + h->B;
    precondition_kernel<<<blocks_for(n, 256), 256, 0, h->stream>>>(h->N, h->B, h->d_rigid, h->d_bsize, x, y);
    CR_LAUNCH(h, "precondition_kernel");
    return CR_OK;
}

// MatrixVectorMultiply (ConductorRigid.cu:953-1020): y = [Phi_b - M q ; S q].
// The wave-space part (spreading, transforms, contraction: L1-, shared-memory- and
// issue-bound, the mesh L2-resident) and the real-space product (bound by its loads in
// flight) are independent given the charges, so unless the profiler is on (its marks
// time one stream) they run side by side: the wave part forks onto the handle's
// high-priority side stream, the real-space product writes its sums, and after the join
// rows_combine_kernel adds the wave part and the self term (the arithmetic of the fused
// form).  In a captured Arnoldi step the fork and join become parallel graph branches.
template <typename R> static int apply_operator_t(cr_handle *h, MeshBuffers<R> &m, const double *x, double *y) {
    CR_TRY(cast_charges(h, m, x));
    if (h->side && !h->prof.on && !(h->rs_onfly & CR_REALSPACE_SERIAL) && h->N > 0) {
        cudaStream_t main = h->stream;
        CR_CUDA(h, cudaEventRecord(h->ev_fork, main));
        CR_CUDA(h, cudaStreamWaitEvent(h->side, h->ev_fork, 0));
        h->stream = h->side;
        int st = wave_potential(h, m);
        if (st == CR_OK) st = check_cuda(h, cudaEventRecord(h->ev_join, h->side), "cudaEventRecord");
        h->stream = main;
        CR_TRY(st);
        const int rs = real_space_apply(h, m, x + h->N, y, true);
        CR_CUDA(h, cudaStreamWaitEvent(main, h->ev_join, 0));  // joins the branch on every path
        CR_TRY(rs);
        CR_TRY(real_space_rows(h, m, x + h->N, y));
    } else {
        CR_TRY(wave_potential(h, m));
        CR_TRY(real_space_apply(h, m, x + h->N, y));
    }
    CR_TRY(body_sums(h, x, y));
    return CR_OK;
}

int apply_operator(cr_handle *h, const double *x, double *y, int precision) {
    if (!h->geo.valid) return fail(h, CR_NOT_READY, "positions not set");
    if (precision == CR_FP64) return apply_operator_t(h, h->m64, x, y);
    return apply_operator_t(h, h->m32, x, y);
}

// ---- lockstep batches: body rows and the diagonal preconditioner ----

namespace {

__global__ void body_sums_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                       const int *__restrict__ mask, int xin, int yout) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &r = reps[it.x];
    const int b = (it.y * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= r.B) return;
    const double *x = r.vec[xin];
    double s = 0.0;
    for (int k = r.body_start[b] + lane; k < r.body_start[b + 1]; k += 32) s += x[r.body_members[k]];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) r.vec[yout][r.N + b] = s;
}

__global__ void diag_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                  const int *__restrict__ mask, int xin, int zout) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &r = reps[it.x];
    const double *x = r.vec[xin];
    double *y = r.vec[zout];
    for (int i = it.y * blockDim.x + threadIdx.x; i < r.n; i += r.vblk * blockDim.x) {
        if (i < r.N) {
            y[i] = -4.0 * kPi * x[i];
        } else {
            const int b = i - r.N;
            y[i] = r.rigid[b] ? x[i] / (double)r.bsize[b] : x[i] / (4.0 * kPi);
        }
    }
}

}  // namespace

int batch_body_sums(cr_batch *bt, const int *mask, int xin, int yout, cudaStream_t s) {
    if (bt->n_items[BL_BODYWARPS] == 0) return CR_OK;
    body_sums_batch_kernel<<<bt->n_items[BL_BODYWARPS], 256, 0, s>>>(bt->d_reps, bt->d_items[BL_BODYWARPS], mask, xin,
                                                                      yout);
    ++bt->launches;
    return batch_check(bt, cudaGetLastError(), "body_sums_batch_kernel");
}

int batch_diag(cr_batch *bt, const int *mask, int xin, int zout, cudaStream_t s) {
    if (bt->n_items[BL_VEC] == 0) return CR_OK;
    diag_batch_kernel<<<bt->n_items[BL_VEC], 256, 0, s>>>(bt->d_reps, bt->d_items[BL_VEC], mask, xin, zout);
    ++bt->launches;
    return batch_check(bt, cudaGetLastError(), "diag_batch_kernel");
}

}  // namespace cr
