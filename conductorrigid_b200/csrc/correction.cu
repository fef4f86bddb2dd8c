// correction.cu -- the learned correction of the preconditioner inside flexible GMRES.
//
// No counterpart in the reference, whose GMRES applies the fixed diagonal scaling of
// Precondition (ConductorRigid.cu:1023-1044, PreconditionWrapper.cuh:63-73) to every
// Krylov vector.  Here the per-bead tensor-core network (mlp.cu) adds a correction to the
// plain preconditioner's output: for a Krylov vector v with z = P v (the handle's
// preconditioner),
//
//     z' = z + weight * s * y(features(v, z)),   s = RMS of z,
//
// where the network reads 48 features per bead -- z_i and v_i scaled to unit RMS, the own
// body's mean and induced dipole of z (projected on the bead's outward direction), the
// field direction, and for the 8 nearest bodies the cosine of the direction to them,
// their proximity, their mean of z and the potential of their induced dipole of z at the
// bead -- and its output y_i corrects bead row i.  The map is homogeneous of degree one
// in v (features are scaled by the RMS of z, the output multiplied by it), as the exact
// inverse is.  Flexible GMRES accepts a preconditioner that changes from step to step,
// so the fixed point A x = b and the stopping test on the true residual are unchanged
// whatever the network outputs.
//
// Training pairs come from solves already done: for a stored preconditioned Krylov
// direction z_j of the last cycle, w = A z_j is a vector whose exact preconditioned
// image A^-1 w = z_j is known, so the target is (z_j - P w) / s at the features of
// (w, P w).
//
// Fallback: before a solve uses the correction it is tried on the solve's initial
// residual r: the one-step least-squares residual over span{A P r} is compared with the
// one over span{A P r, A c} (c the correction of r), and the correction is used in that
// solve only if it lowers that residual by at least 1 % -- at the scale the least-squares
// fit gives it;
// otherwise the solve runs with the plain preconditioner alone.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "cr_internal.cuh"

namespace cr {

int mlp_forward_async(cr_mlp *h, int n, const uint16_t *d_x, float *d_y, cudaStream_t s);
int mlp_check(cr_mlp *h, cudaStream_t s);

namespace {

constexpr int KN = 8;                  // nearest bodies in the features
constexpr int NF = CR_MLP_FEATURES;    // 48

__device__ inline double mimg(double d, double L) { return d - L * rint(d / L); }

// KN nearest other bodies of every body by centre distance (minimum image; ties by lower
// index; missing entries point at the body itself).
__global__ void nearest_bodies_kernel(int B, const double4 *__restrict__ bpos, double Lx, double Ly, double Lz,
                                      int *__restrict__ nbr) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    double best[KN];
    int idx[KN];
    for (int k = 0; k < KN; ++k) {
        best[k] = 1e300;
        idx[k] = b;
    }
    const double4 c = bpos[b];
    for (int j = 0; j < B; ++j) {
        if (j == b) continue;
        const double4 o = bpos[j];
        const double dx = mimg(o.x - c.x, Lx), dy = mimg(o.y - c.y, Ly), dz = mimg(o.z - c.z, Lz);
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 >= best[KN - 1]) continue;
        int p = KN - 1;
        while (p > 0 && best[p - 1] > d2) {
            best[p] = best[p - 1];
            idx[p] = idx[p - 1];
            --p;
        }
        best[p] = d2;
        idx[p] = j;
    }
    for (int k = 0; k < KN; ++k) nbr[(size_t)b * KN + k] = idx[k];
}

// Per body: mean of z over its beads and the induced dipole sum_j z_j (r_j - R_b)
// (minimum image); mom[b] = (mean, dx, dy, dz).  One warp per body.
__global__ void body_moments_kernel(int B, const int *__restrict__ start, const int *__restrict__ members,
                                    const double4 *__restrict__ pos, const double4 *__restrict__ bpos, double Lx,
                                    double Ly, double Lz, const double *__restrict__ z, double4 *__restrict__ mom) {
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= B) return;
    const double4 c = bpos[b];
    const int k0 = start[b], k1 = start[b + 1];
    double s = 0, dx = 0, dy = 0, dz = 0;
    for (int k = k0 + lane; k < k1; k += 32) {
        const int i = members[k];
        const double4 p = pos[i];
        const double zi = z[i];
        s += zi;
        dx += zi * mimg(p.x - c.x, Lx);
        dy += zi * mimg(p.y - c.y, Ly);
        dz += zi * mimg(p.z - c.z, Lz);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        dx += __shfl_xor_sync(0xffffffffu, dx, o);
        dy += __shfl_xor_sync(0xffffffffu, dy, o);
        dz += __shfl_xor_sync(0xffffffffu, dz, o);
    }
    if (lane == 0) mom[b] = make_double4(k1 > k0 ? s / (double)(k1 - k0) : 0.0, dx, dy, dz);
}

__device__ inline uint32_t bf16(float a) {
    __nv_bfloat16 v = __float2bfloat16_rn(a);
    return (uint32_t)(*reinterpret_cast<uint16_t *>(&v));
}

struct FeatGeom {
    double L[3];
    double E0[3];
    int N, n;  // beads, unknowns (N + B)
};

// 48 BF16 features of every bead for the vector pair (v, z); ss[0] = |z|^2, ss[1] = |v|^2
// over all n unknowns (RMS scales sqrt(ss / n)).
__global__ void corr_features_kernel(FeatGeom g, const uint32_t *__restrict__ body, const double4 *__restrict__ pos,
                                     const double4 *__restrict__ bpos, const int *__restrict__ nbr,
                                     const double4 *__restrict__ mom, const double *__restrict__ v,
                                     const double *__restrict__ z, const double *__restrict__ ss,
                                     uint16_t *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    const double sz = sqrt(ss[0] / g.n), sv = sqrt(ss[1] / g.n);
    const double iz = sz > 0 ? 1.0 / sz : 0.0, iv = sv > 0 ? 1.0 / sv : 0.0;
    const int b = body[i];
    const double4 p = pos[i], c = bpos[b], mb = mom[b];
    double nx = mimg(p.x - c.x, g.L[0]), ny = mimg(p.y - c.y, g.L[1]), nz = mimg(p.z - c.z, g.L[2]);
    const double rn = sqrt(nx * nx + ny * ny + nz * nz);
    if (rn > 0) {
        nx /= rn;
        ny /= rn;
        nz /= rn;
    }
    float f[NF];
    f[0] = (float)(z[i] * iz);
    f[1] = (float)(v[i] * iv);
    f[2] = (float)(mb.x * iz);
    f[3] = (float)((z[i] - mb.x) * iz);
    f[4] = (float)((mb.y * nx + mb.z * ny + mb.w * nz) * iz);
    f[5] = (float)(sqrt(mb.y * mb.y + mb.z * mb.z + mb.w * mb.w) * iz);
    f[6] = (float)(g.E0[0] * nx + g.E0[1] * ny + g.E0[2] * nz);
    f[7] = 0.f;
    for (int k = 0; k < KN; ++k) {
        const int o = nbr[(size_t)b * KN + k];
        float *ff = f + 8 + 5 * k;
        if (o == b) {
            ff[0] = ff[1] = ff[2] = ff[3] = ff[4] = 0.f;
            continue;
        }
        const double4 co = bpos[o], mo = mom[o];
        // from the bead to body o's centre
        const double ux = mimg(co.x - p.x, g.L[0]), uy = mimg(co.y - p.y, g.L[1]), uz = mimg(co.z - p.z, g.L[2]);
        const double D = sqrt(ux * ux + uy * uy + uz * uz);
        const double inv = D > 0 ? 1.0 / D : 0.0;
        const double cosv = (nx * ux + ny * uy + nz * uz) * inv;
        const double prox = 1.0 / (1.0 + D);
        // potential at the bead of body o's induced dipole: d . (r_i - R_o) / |r_i - R_o|^3
        const double dip = -(mo.y * ux + mo.z * uy + mo.w * uz) * inv * inv * inv;
        ff[0] = (float)cosv;
        ff[1] = (float)prox;
        ff[2] = (float)(mo.x * iz);
        ff[3] = (float)(dip * iz);
        ff[4] = (float)(prox * cosv);
    }
    uint16_t *row = out + (size_t)i * NF;
#pragma unroll
    for (int k = 0; k < NF; k += 8) {
        uint4 w;
        w.x = bf16(f[k]) | (bf16(f[k + 1]) << 16);
        w.y = bf16(f[k + 2]) | (bf16(f[k + 3]) << 16);
        w.z = bf16(f[k + 4]) | (bf16(f[k + 5]) << 16);
        w.w = bf16(f[k + 6]) | (bf16(f[k + 7]) << 16);
        *reinterpret_cast<uint4 *>(row + k) = w;
    }
}

// z_i += weight * s * y_i on the bead rows (s = RMS of z before the correction)
__global__ void corr_apply_kernel(int N, int n, double weight, const double *__restrict__ ss,
                                  const float *__restrict__ y, double *__restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    z[i] += weight * sqrt(ss[0] / n) * (double)y[i];
}

// t_i = (zt_i - zp_i) / s, s = RMS of zp
__global__ void corr_target_kernel(int N, int n, const double *__restrict__ zt, const double *__restrict__ zp,
                                   const double *__restrict__ ss, float *__restrict__ t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double s = sqrt(ss[0] / n);
    t[i] = s > 0 ? (float)((zt[i] - zp[i]) / s) : 0.f;
}

FeatGeom feat_geom(const cr_handle *h) {
    FeatGeom g;
    for (int d = 0; d < 3; ++d) {
        g.L[d] = h->L[d];
        g.E0[d] = h->field[d];
    }
    g.N = h->N;
    g.n = h->N + h->B;
    return g;
}

// BF16 feature rows of (v, z) into out (z is the plain preconditioner's output for v).
int correction_features(cr_handle *h, const double *v, const double *z, uint16_t *out) {
    Correction &c = h->corr;
    CR_TRY(dots(h, 1, z, z, c.ss));
    CR_TRY(dots(h, 1, v, v, c.ss + 1));
    if (h->B > 0) {
        body_moments_kernel<<<blocks_for((long)h->B * 32, 256), 256, 0, h->stream>>>(
            h->B, h->d_body_start, h->d_body_members, h->m64.pos, h->d_bpos, h->L[0], h->L[1], h->L[2], z, c.mom);
        CR_LAUNCH(h, "body_moments_kernel");
    }
    corr_features_kernel<<<blocks_for(h->N, 128), 128, 0, h->stream>>>(feat_geom(h), h->d_body, h->m64.pos,
                                                                        h->d_bpos, c.nbr, c.mom, v, z, c.ss, out);
    CR_LAUNCH(h, "corr_features_kernel");
    return CR_OK;
}

}  // namespace

// Buffers and the nearest-body lists of the current geometry (outside any capture).
int correction_prepare(cr_handle *h) {
    Correction &c = h->corr;
    if (!c.net || h->N == 0) return CR_OK;
    if (c.cap_n != h->N || c.cap_b != h->B) {
        CR_TRY(dalloc(h, &c.x, (size_t)h->N * NF));
        CR_TRY(dalloc(h, &c.y, (size_t)h->N));
        CR_TRY(dalloc(h, &c.nbr, (size_t)std::max(h->B, 1) * KN));
        CR_TRY(dalloc(h, &c.mom, (size_t)std::max(h->B, 1)));
        CR_TRY(dalloc(h, &c.ss, 2));
        CR_TRY(dalloc(h, &c.zp, (size_t)(h->N + h->B)));
        CR_TRY(dalloc(h, &c.zc, (size_t)(h->N + h->B)));
        c.cap_n = h->N;
        c.cap_b = h->B;
        c.nbr_gen = -1;
    }
    if (c.nbr_gen != h->geo_gen && h->B > 0) {
        nearest_bodies_kernel<<<blocks_for(h->B, 128), 128, 0, h->stream>>>(h->B, h->d_bpos, h->L[0], h->L[1],
                                                                           h->L[2], c.nbr);
        CR_LAUNCH(h, "nearest_bodies_kernel");
        c.nbr_gen = h->geo_gen;
    }
    return CR_OK;
}

void correction_free(cr_handle *h) {
    Correction &c = h->corr;
    dfree(&c.x);
    dfree(&c.y);
    dfree(&c.nbr);
    dfree(&c.mom);
    dfree(&c.ss);
    dfree(&c.zp);
    dfree(&c.zc);
    c.cap_n = c.cap_b = -1;
    c.nbr_gen = -1;
}

// z += weight * s * network(features(v, z)); no host synchronisation (capturable).
int correction_add(cr_handle *h, const double *v, double *z) {
    Correction &c = h->corr;
    CR_TRY(correction_features(h, v, z, c.x));
    if (mlp_forward_async(c.net, h->N, c.x, c.y, h->stream) != CR_OK)
        return fail(h, CR_CUDA_ERROR, "learned correction: network launch failed");
    corr_apply_kernel<<<blocks_for(h->N, 256), 256, 0, h->stream>>>(h->N, h->N + h->B, c.weight * c.scale, c.ss,
                                                                     c.y, z);
    CR_LAUNCH(h, "corr_apply_kernel");
    return CR_OK;
}

// The preconditioner of one flexible-GMRES step: the handle's plain preconditioner, plus
// the learned correction when the current solve uses it.
int precondition_step(cr_handle *h, const double *v, double *z) {
    CR_TRY(precondition(h, v, z));
    if (h->corr.active) CR_TRY(correction_add(h, v, z));
    return CR_OK;
}

// Decide for this solve (residual r, operator precision `precision`): with zp = P r and
// c the network's correction of r (at the caller's weight), the one-step least-squares
// residual over span{A zp} and over span{A zp, A c}.  The correction is used only if the
// second is smaller by at least 1 %, and then with the fitted scale: the solve's steps apply
// zp + (a_c / a_p) c, (a_p, a_c) the least-squares coefficients.
int correction_decide(cr_handle *h, int precision, const double *r, double *w) {
    Correction &c = h->corr;
    c.active = 0;
    c.scale = 1.0;
    c.last_rho[0] = c.last_rho[1] = -1.0;
    if (!c.net || c.weight == 0.0 || h->N == 0) return CR_OK;
    CR_TRY(correction_prepare(h));
    const int n = h->N + h->B;
    CR_TRY(precondition(h, r, c.zp));
    CR_CUDA(h, cudaMemsetAsync(c.zc, 0, (size_t)n * sizeof(double), h->stream));
    CR_TRY(correction_features(h, r, c.zp, c.x));  // the correction alone, into zc
    if (mlp_forward_async(c.net, h->N, c.x, c.y, h->stream) != CR_OK)
        return fail(h, CR_CUDA_ERROR, "learned correction: network launch failed");
    corr_apply_kernel<<<blocks_for(h->N, 256), 256, 0, h->stream>>>(h->N, n, c.weight, c.ss, c.y, c.zc);
    CR_LAUNCH(h, "corr_apply_kernel");
    Krylov &K = h->kry;
    double *wp = w, *wc = K.d;  // A zp and A c (K.d is free before the solve's refinement)
    CR_TRY(apply_operator(h, c.zp, wp, precision));
    CR_TRY(apply_operator(h, c.zc, wc, precision));
    CR_TRY(dots(h, 1, r, r, K.hcol));
    CR_TRY(dots(h, 1, wp, r, K.hcol + 1));
    CR_TRY(dots(h, 1, wc, r, K.hcol + 2));
    double g[3];
    CR_TRY(dots(h, 1, wp, wp, K.hcol + 3));
    CR_TRY(dots(h, 1, wp, wc, K.hcol + 4));
    CR_TRY(dots(h, 1, wc, wc, K.hcol + 5));
    CR_CUDA(h, cudaMemcpyAsync(K.h_pinned, K.hcol, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    if (mlp_check(c.net, h->stream) != CR_OK) return fail(h, CR_TIMEOUT, "learned correction: network wait ran out");
    const double rr = K.h_pinned[0], pr = K.h_pinned[1], cr = K.h_pinned[2];
    g[0] = K.h_pinned[3];
    g[1] = K.h_pinned[4];
    g[2] = K.h_pinned[5];
    if (!(rr > 0) || !(g[0] > 0)) return CR_OK;
    const double rho_p = std::max(0.0, 1.0 - pr * pr / (rr * g[0]));
    c.last_rho[0] = std::sqrt(rho_p);
    const double det = g[0] * g[2] - g[1] * g[1];
    if (!(det > 1e-12 * g[0] * g[2])) {  // the correction adds no new direction
        c.last_rho[1] = c.last_rho[0];
        return CR_OK;
    }
    const double ap = (g[2] * pr - g[1] * cr) / det, ac = (g[0] * cr - g[1] * pr) / det;
    const double rho_c = std::max(0.0, 1.0 - (ap * pr + ac * cr) / rr);
    c.last_rho[1] = std::sqrt(rho_c);
    // a direction unrelated to r lowers the least-squares residual by ~1/n only: the
    // correction must lower it by at least 1 % to be used
    if (std::isfinite(rho_c) && ap != 0.0 && std::isfinite(ac / ap) && c.last_rho[1] < 0.99 * c.last_rho[0]) {
        c.active = 1;
        c.scale = ac / ap;
    }
    return CR_OK;
}

// Training rows from the last solve's stored directions: for up to max_dirs columns z_j
// of the last Krylov cycle, w = A z_j (FP64), features of (w, P w) into d_x and targets
// (z_j - P w) / s into d_t, N rows per direction.
int correction_samples(cr_handle *h, int max_dirs, uint16_t *d_x, float *d_t, int *rows) {
    Correction &c = h->corr;
    *rows = 0;
    Krylov &K = h->kry;
    const int k = std::min(max_dirs, K.last_cols);
    if (k <= 0 || h->N == 0) return CR_OK;
    CR_TRY(correction_prepare(h));
    const int n = h->N + h->B;
    for (int j = 0; j < k; ++j) {
        const double *zt = K.Z + (size_t)j * n;
        CR_TRY(apply_operator(h, zt, c.zc, CR_FP64));
        CR_TRY(precondition(h, c.zc, c.zp));
        CR_TRY(correction_features(h, c.zc, c.zp, d_x + (size_t)j * h->N * NF));
        corr_target_kernel<<<blocks_for(h->N, 256), 256, 0, h->stream>>>(h->N, n, zt, c.zp, c.ss,
                                                                         d_t + (size_t)j * h->N);
        CR_LAUNCH(h, "corr_target_kernel");
    }
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    *rows = k * h->N;
    return CR_OK;
}

}  // namespace cr
