// realspace.cu -- real-space part of the operator and of the force pass
// (ConductorRigid.cu:469-664).
//
// One warp per bead walks its neighbour list (built once per solve within rc); lanes
// stride over the neighbours, gather positions and charges through the read-only
// cache, apply the minimum image (ConductorRigid.cu:536), the cutoff window
// dr^2 <= d^2 < rc^2 (cu:540) and the tabulated, linearly interpolated kernel
// (index floor(Ntable (d - dr)/(rc - dr)), weight d/dr - index - 1, cu:549-554).  The
// index is clamped to the table so that rounding at either end of the window never
// reads outside it.
#include "cr_internal.cuh"

namespace cr {

namespace {

template <typename R> struct RSConst {
    R L[3], Linv[3];
    R rc2, rmin2, dr, inv_dr, tab_scale;  // tab_scale = Ntable / (rc - dr)
    int ntab;
    R selfc;
    R E0[3];
};

__device__ __forceinline__ float rint_r(float x) { return rintf(x); }
__device__ __forceinline__ double rint_r(double x) { return rint(x); }
__device__ __forceinline__ float floor_r(float x) { return floorf(x); }
__device__ __forceinline__ double floor_r(double x) { return floor(x); }
__device__ __forceinline__ float sqrt_r(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_r(double x) { return sqrt(x); }

template <typename R> __device__ __forceinline__ R warp_sum(R v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename R> __device__ __forceinline__ R table_lerp(const typename Prec<R>::R2 *tab, const RSConst<R> &c, R d) {
    int ind = (int)floor_r((d - c.dr) * c.tab_scale);
    ind = min(max(ind, 0), c.ntab - 1);
    const R lin = d * c.inv_dr - (R)ind - (R)1;
    const typename Prec<R>::R2 e = __ldg(tab + ind);
    return e.x + (e.y - e.x) * lin;
}

// out_i = Phi_body(i) - (phik_i + self q_i + sum_j T(d_ij) q_j)   (phi_body != NULL)
// out_i = phik_i + self q_i + sum_j T(d_ij) q_j                   (phi_body == NULL)
template <typename R>
__global__ void __launch_bounds__(256) real_potential_kernel(
    int N, const typename Prec<R>::R4 *__restrict__ pos, const R *__restrict__ q, const int *__restrict__ count,
    const int64_t *__restrict__ head, const int *__restrict__ list, const typename Prec<R>::R2 *__restrict__ tab,
    RSConst<R> c, const R *__restrict__ phik, const double *__restrict__ phi_body, const uint32_t *__restrict__ body,
    double *__restrict__ out) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    const typename Prec<R>::R4 pi = pos[i];
    const int64_t h0 = head[i];
    const int n = count[i];
    R acc = 0;
    for (int k = lane; k < n; k += 32) {
        const int j = __ldg(list + h0 + k);
        const typename Prec<R>::R4 pj = pos[j];
        R dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        dx -= c.L[0] * rint_r(dx * c.Linv[0]);
        dy -= c.L[1] * rint_r(dy * c.Linv[1]);
        dz -= c.L[2] * rint_r(dz * c.Linv[2]);
        const R d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < c.rc2 && d2 >= c.rmin2) acc += table_lerp<R>(tab, c, sqrt_r(d2)) * __ldg(q + j);
    }
    acc = warp_sum(acc);
    if (lane == 0) {
        const double total = (double)phik[i] + (double)(c.selfc * q[i]) + (double)acc;
        out[i] = phi_body ? phi_body[body[i]] - total : total;
    }
}

// force_i = wave force_i + q_i E0 + sum_j -T'(d_ij) q_i q_j rhat_ij   (cu:596-662)
template <typename R>
__global__ void __launch_bounds__(256) real_force_kernel(
    int N, const typename Prec<R>::R4 *__restrict__ pos, const R *__restrict__ q, const int *__restrict__ count,
    const int64_t *__restrict__ head, const int *__restrict__ list, const typename Prec<R>::R2 *__restrict__ tab,
    RSConst<R> c, const R *__restrict__ fk, double *__restrict__ out) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    const typename Prec<R>::R4 pi = pos[i];
    const int64_t h0 = head[i];
    const int n = count[i];
    R fx = 0, fy = 0, fz = 0;
    for (int k = lane; k < n; k += 32) {
        const int j = __ldg(list + h0 + k);
        const typename Prec<R>::R4 pj = pos[j];
        R dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        dx -= c.L[0] * rint_r(dx * c.Linv[0]);
        dy -= c.L[1] * rint_r(dy * c.Linv[1]);
        dz -= c.L[2] * rint_r(dz * c.Linv[2]);
        const R d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < c.rc2 && d2 >= c.rmin2) {
            const R d = sqrt_r(d2);
            const R a = table_lerp<R>(tab, c, d) * __ldg(q + j) / d;
            fx -= a * dx;
            fy -= a * dy;
            fz -= a * dz;
        }
    }
    fx = warp_sum(fx);
    fy = warp_sum(fy);
    fz = warp_sum(fz);
    if (lane == 0) {
        const R qi = q[i];
        out[3 * (size_t)i + 0] = (double)fk[3 * (size_t)i + 0] + (double)(qi * c.E0[0]) + (double)(qi * fx);
        out[3 * (size_t)i + 1] = (double)fk[3 * (size_t)i + 1] + (double)(qi * c.E0[1]) + (double)(qi * fy);
        out[3 * (size_t)i + 2] = (double)fk[3 * (size_t)i + 2] + (double)(qi * c.E0[2]) + (double)(qi * fz);
    }
}

template <typename R> RSConst<R> rs_const(const cr_handle *h) {
    RSConst<R> c;
    for (int d = 0; d < 3; ++d) {
        c.L[d] = (R)h->L[d];
        c.Linv[d] = (R)(1.0 / h->L[d]);
        c.E0[d] = (R)h->field[d];
    }
    c.rc2 = (R)(h->d.rcut * h->d.rcut);
    c.rmin2 = (R)(h->d.dr * h->d.dr);
    c.dr = (R)h->d.dr;
    c.inv_dr = (R)(1.0 / h->d.dr);
    c.tab_scale = (R)(h->d.n_table / (h->d.rcut - h->d.dr));
    c.ntab = h->d.n_table;
    c.selfc = (R)h->d.selfcoeff;
    return c;
}

}  // namespace

template <typename R> int real_space_apply(cr_handle *h, MeshBuffers<R> &m, const double *phi_body, double *out) {
    const int N = h->N;
    if (N == 0) return CR_OK;
    ProfScope ps(h, PROF_REAL);
    real_potential_kernel<R><<<blocks_for((long)N * 32, 256), 256, 0, h->stream>>>(
        N, m.pos, m.q, h->geo.nl_count, h->geo.nl_head, h->geo.nl_list, m.phiq, rs_const<R>(h), m.phi, phi_body,
        h->d_body, out);
    CR_LAUNCH(h, "real_potential_kernel");
    return CR_OK;
}

template <typename R> int real_space_force(cr_handle *h, MeshBuffers<R> &m, double *force_out) {
    const int N = h->N;
    if (N == 0) return CR_OK;
    ProfScope ps(h, PROF_REAL_FORCE);
    real_force_kernel<R><<<blocks_for((long)N * 32, 256), 256, 0, h->stream>>>(
        N, m.pos, m.q, h->geo.nl_count, h->geo.nl_head, h->geo.nl_list, m.gradphiq, rs_const<R>(h), m.force,
        force_out);
    CR_LAUNCH(h, "real_force_kernel");
    return CR_OK;
}

template int real_space_apply<float>(cr_handle *, MeshBuffers<float> &, const double *, double *);
template int real_space_apply<double>(cr_handle *, MeshBuffers<double> &, const double *, double *);
template int real_space_force<float>(cr_handle *, MeshBuffers<float> &, double *);
template int real_space_force<double>(cr_handle *, MeshBuffers<double> &, double *);

}  // namespace cr
