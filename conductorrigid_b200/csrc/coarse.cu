// coarse.cu -- two-level conductor preconditioner (CR_PRECOND_TWO_LEVEL).
//
// The conductor response (conductor.cu) inverts every body's own block exactly; what it
// leaves to the Krylov iteration are the collective modes in which whole bodies polarise
// one another (chains of nearly touching conductors at high volume fraction).  Those
// modes live, to a good approximation, in the span of the bodies' induced dipoles, so a
// coarse space of three vectors per body is added:
//
//   z_ba = A_b^-1 [ -(r - r_b0).e_a ; 0 ]      a = x, y, z,
//
// the charges the isolated conductor b carries in a unit external field along a (A_b
// the body block of conductor.cu, r_b0 its first bead).  The columns are neutral
// (1^T q = 0), so on them the constraint rows of the saddle-point operator vanish and the
// coarse operator is C = -Z^T A~ Z = Z_q^T M~ Z_q, symmetric positive definite, with
// the model operator M~ = the exact self and real-space terms plus the wave-space term
// truncated to |k| < kc = 2 xi:
//
//   Z_q^T M~_wave Z_q = sum_{k in the half space, 0 < |k| < kc} w_k Re[S_a(k) conj S_b(k)],
//   S_a(k) = sum_{i in a} z_a(i) exp(-i k.r_i),   w_k = 2 j0(|k|)^2 exp(-k^2/4xi^2) / (k^2 V),
//
// the low-k part of the reference's wave-space kernel (ConductorRigid.cc:245-274: the
// shell form factor j0^2 and the Ewald factor, here without the spreading windows it
// divides out).  The correction is applied in the A-DEF1 form of deflation (Tang, Nabben,
// Vuik and Erlangga, J. Sci. Comput. 39, 2009):
//
//   y = A_c^-1 Z^T r = -C^-1 Z^T r,      z = P (r - A~ Z y) + Z y,
//
// P the conductor response.  A~ Z y = [Phi(Z y) - M~ Z_q y ; 0] is evaluated from blocks
// W = M_real Z_q stored per pair of near bodies and from the same k-sum; C^-1 is formed
// once per geometry (assembled in FP64, inverted in place by blocked Gauss-Jordan in FP32).
// Above a dense limit (max_dense coarse unknowns, 12,288 by default) the level is skipped
// unless the caller asks for the sparse form (cr_set_coarse with CG steps > 0): the coarse
// operator is then kept as 3 x 3 blocks of the near pairs plus the low-rank F F^T (at most
// 256 wave vectors), and C y = -Z^T r is solved by that many block-Jacobi preconditioned
// CG steps.
// In flexible GMRES any preconditioner leaves the solution unchanged: only the iteration
// count moves (at 162 beads per sphere, phi = 0.30: 133 -> 40 iterations against the
// conductor response alone, on 100 bodies).
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "cr_internal.cuh"

namespace cr {

namespace {

constexpr int kMinBeads = 4;        // bodies with fewer beads get no coarse vectors
constexpr int kMaxSparse = 786432;  // coarse unknowns above which the level is skipped
constexpr int kMaxModes = 1024;     // half-space wave vectors kept (kc shrinks above)
constexpr int kMaxModesSparse = 256;  // the same for the sparse form (its CG steps read F twice)
constexpr int NB = 64;              // Gauss-Jordan block
constexpr int GT = 128;             // Gauss-Jordan update tile; the padded order is a multiple of it
constexpr int kChunk = 512;         // beads staged in shared memory per pass

__device__ __forceinline__ double mimgd(double d, double L, double Linv) { return d - L * rint(d * Linv); }
__device__ __forceinline__ float mimgf(float d, float L, float Linv) { return d - L * rintf(d * Linv); }

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *red /* [NV][32] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int t = 0; t < NV; ++t) {
        double s = v[t];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[t * 32 + warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int t = 0; t < NV; ++t) {
            double s = lane < nw ? red[t * 32 + lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            v[t] = s;  // valid in thread 0
        }
    }
    __syncthreads();
}

// Right-hand sides of the three basis solves: x_a[i] = -(r_i - r_b0).e_a, 0 on body rows.
__global__ void basis_rhs_kernel(int N, int B, const uint32_t *__restrict__ body, const int *__restrict__ body_start,
                                 const int *__restrict__ members, const double4 *__restrict__ pos, double3 L,
                                 double3 Linv, double *__restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = N + B;
    if (i >= n) return;
    if (i >= N) {
        x[i] = x[n + i] = x[2 * n + i] = 0.0;
        return;
    }
    const double4 p = pos[i], p0 = pos[members[body_start[body[i]]]];
    x[i] = -mimgd(p.x - p0.x, L.x, Linv.x);
    x[n + i] = -mimgd(p.y - p0.y, L.y, Linv.y);
    x[2 * n + i] = -mimgd(p.z - p0.z, L.z, Linv.z);
}

// Basis of the coarse bodies (zeros elsewhere), their centroid and bounding radius.
__global__ void basis_pack_kernel(int N, int B, const int *__restrict__ body_start, const int *__restrict__ members,
                                  const int *__restrict__ cidx, const double4 *__restrict__ pos, double3 L,
                                  double3 Linv, const double *__restrict__ y, double *__restrict__ zq,
                                  double *__restrict__ zp, double4 *__restrict__ cent) {
    __shared__ double red[4 * 32];
    const int b = blockIdx.x;
    const int n = N + B;
    const int beg = body_start[b], nb = body_start[b + 1] - beg;
    if (nb == 0) {  // a body without beads: no columns, centre never read
        if (threadIdx.x < 3) zp[3 * b + threadIdx.x] = 0.0;
        if (threadIdx.x == 0) cent[b] = make_double4(0.0, 0.0, 0.0, 0.0);
        return;
    }
    const bool on = cidx[b] >= 0;
    const double4 p0 = pos[members[beg]];
    double s[3] = {0.0, 0.0, 0.0};
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        const int i = members[beg + k];
        for (int a = 0; a < 3; ++a) zq[3 * i + a] = on ? y[a * n + i] : 0.0;
        const double4 p = pos[i];
        s[0] += mimgd(p.x - p0.x, L.x, Linv.x);
        s[1] += mimgd(p.y - p0.y, L.y, Linv.y);
        s[2] += mimgd(p.z - p0.z, L.z, Linv.z);
    }
    block_sum<3>(s, red);
    __shared__ double c[3];
    if (threadIdx.x == 0)
        for (int a = 0; a < 3; ++a) c[a] = s[a] / nb;
    __syncthreads();
    double r2[1] = {0.0};
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        const double4 p = pos[members[beg + k]];
        const double dx = mimgd(p.x - p0.x, L.x, Linv.x) - c[0];
        const double dy = mimgd(p.y - p0.y, L.y, Linv.y) - c[1];
        const double dz = mimgd(p.z - p0.z, L.z, Linv.z) - c[2];
        r2[0] = fmax(r2[0], dx * dx + dy * dy + dz * dz);
    }
    // max-reduce through the sum helper's shared scratch
    for (int o = 16; o > 0; o >>= 1) r2[0] = fmax(r2[0], __shfl_xor_sync(0xffffffffu, r2[0], o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = r2[0];
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        cent[b] = make_double4(mimgd(p0.x + c[0], L.x, Linv.x), mimgd(p0.y + c[1], L.y, Linv.y),
                               mimgd(p0.z + c[2], L.z, Linv.z), sqrt(m));
        for (int a = 0; a < 3; ++a) zp[3 * b + a] = on ? y[a * n + N + b] : 0.0;
    }
}

// Near body pairs (a, b) of coarse bodies, both orders and a == b: one warp per a scans
// every b; FILL writes b in ascending order, so the lists do not depend on scheduling.
template <bool FILL>
__global__ void near_pairs_kernel(int nbc, const int *__restrict__ cbody, const double4 *__restrict__ cent,
                                  double3 L, double3 Linv, double rc, int *__restrict__ count,
                                  const int *__restrict__ head, int *__restrict__ pair_b) {
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (a >= nbc) return;
    const double4 ca = cent[cbody[a]];
    int n = 0;
    const int h0 = FILL ? head[a] : 0;
    for (int base = 0; base < nbc; base += 32) {
        const int b = base + lane;
        bool hit = false;
        if (b < nbc) {
            const double4 cb = cent[cbody[b]];
            const double dx = mimgd(cb.x - ca.x, L.x, Linv.x), dy = mimgd(cb.y - ca.y, L.y, Linv.y),
                         dz = mimgd(cb.z - ca.z, L.z, Linv.z);
            const double reach = rc + ca.w + cb.w;
            hit = dx * dx + dy * dy + dz * dz < reach * reach;
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (FILL && hit) pair_b[h0 + n + __popc(m & ((1u << lane) - 1u))] = b;
        n += __popc(m);
    }
    if (!FILL && lane == 0) count[a] = n;
}

// T(d) from the FP32 table with the reference's index and weight (ConductorRigid.cu:549-554):
// index floor((d - dr) ntab / (rc - dr)) (scale = ntab / (rc - dr)), weight d/dr - index - 1.
__device__ __forceinline__ float table_lerp32(const float2 *__restrict__ tab, int ntab, float scale, float dr,
                                              float inv_dr, float d) {
    const int ind = min(max((int)((d - dr) * scale), 0), ntab - 1);
    const float lin = fmaf(d, inv_dr, -1.0f) - (float)ind;
    const float2 e = __ldg(tab + ind);
    return fmaf(e.y - e.x, lin, e.x);
}

struct RealArgs {
    double Ld[3];
    float L[3], Linv[3];
    float rc, rc2, rmin2, dr, inv_dr, scale;
    int ntab;
    double selfc;
};

// One CTA per ordered near pair p = (a, b):  W_p[k][c] = sum_{j in b} T(d_kj) z_bc(j) for
// the beads k of a (the operator's pair rule dr <= d < rc under the minimum image), and
// C[3a+e][3b+c] += sum_k z_ae(k) W_p[k][c] (+ the self term when a == b).
// SHIFT (boxes of edge >= 2 (rc + 2 max radius)): every bead pair of two near bodies takes
// the image of the centroids' minimum image, so positions are staged relative to a's
// centroid once per bead and the pair loop needs no minimum image; otherwise each bead
// pair takes its own.
template <bool SHIFT>
__global__ void __launch_bounds__(256) coarse_real_kernel(
    const int *__restrict__ pair_a, const int *__restrict__ pair_b, const long long *__restrict__ woff,
    const int *__restrict__ cbody, const int *__restrict__ body_start, const int *__restrict__ members,
    const double4 *__restrict__ pos, const double4 *__restrict__ cent, const double *__restrict__ zq,
    const float2 *__restrict__ tab, RealArgs g, int ldc, float *__restrict__ W, double *__restrict__ C,
    double *__restrict__ Cblk) {
    __shared__ float4 sp[kChunk];
    __shared__ float2 sz[kChunk];
    __shared__ double red[9 * 32];
    const int p = blockIdx.x;
    const int a = pair_a[p], b = pair_b[p];
    const int ba = cbody[a], bb = cbody[b];
    const int abeg = body_start[ba], na = body_start[ba + 1] - abeg;
    const int bbeg = body_start[bb], nbb = body_start[bb + 1] - bbeg;
    const double4 ca = cent[ba], cb = cent[bb];
    const double Ld[3] = {g.Ld[0], g.Ld[1], g.Ld[2]}, Li[3] = {1.0 / g.Ld[0], 1.0 / g.Ld[1], 1.0 / g.Ld[2]};
    // b's centroid in the image nearest a's, relative to a's
    const double sh[3] = {mimgd(cb.x - ca.x, Ld[0], Li[0]), mimgd(cb.y - ca.y, Ld[1], Li[1]),
                          mimgd(cb.z - ca.z, Ld[2], Li[2])};
    double cacc[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) cacc[t] = 0.0;
    for (int k0 = 0; k0 < na; k0 += blockDim.x) {
        const int k = k0 + threadIdx.x;
        float3 pi = make_float3(0.f, 0.f, 0.f);
        float zi[3] = {0.f, 0.f, 0.f};
        if (k < na) {
            const int i = members[abeg + k];
            const double4 q = pos[i];
            if (SHIFT)
                pi = make_float3((float)mimgd(q.x - ca.x, Ld[0], Li[0]), (float)mimgd(q.y - ca.y, Ld[1], Li[1]),
                                 (float)mimgd(q.z - ca.z, Ld[2], Li[2]));
            else
                pi = make_float3((float)q.x, (float)q.y, (float)q.z);
            for (int c = 0; c < 3; ++c) zi[c] = (float)zq[3 * i + c];
        }
        float acc[3] = {0.f, 0.f, 0.f};
        for (int j0 = 0; j0 < nbb; j0 += kChunk) {
            const int nj = min(kChunk, nbb - j0);
            __syncthreads();
            for (int t = threadIdx.x; t < nj; t += blockDim.x) {
                const int j = members[bbeg + j0 + t];
                const double4 q = pos[j];
                float3 r;
                if (SHIFT)
                    r = make_float3((float)(mimgd(q.x - cb.x, Ld[0], Li[0]) + sh[0]),
                                    (float)(mimgd(q.y - cb.y, Ld[1], Li[1]) + sh[1]),
                                    (float)(mimgd(q.z - cb.z, Ld[2], Li[2]) + sh[2]));
                else
                    r = make_float3((float)q.x, (float)q.y, (float)q.z);
                sp[t] = make_float4(r.x, r.y, r.z, (float)zq[3 * j]);
                sz[t] = make_float2((float)zq[3 * j + 1], (float)zq[3 * j + 2]);
            }
            __syncthreads();
            if (k < na) {
                for (int t = 0; t < nj; ++t) {
                    const float4 q = sp[t];
                    float dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
                    if (!SHIFT) {
                        dx = mimgf(dx, g.L[0], g.Linv[0]);
                        dy = mimgf(dy, g.L[1], g.Linv[1]);
                        dz = mimgf(dz, g.L[2], g.Linv[2]);
                    }
                    const float d2 = dx * dx + dy * dy + dz * dz;
                    if (d2 < g.rc2 && d2 >= g.rmin2) {
                        const float T = table_lerp32(tab, g.ntab, g.scale, g.dr, g.inv_dr, d2 * rsqrtf(d2));
                        const float2 z12 = sz[t];
                        acc[0] += T * q.w;
                        acc[1] += T * z12.x;
                        acc[2] += T * z12.y;
                    }
                }
            }
        }
        if (k < na) {
            float *w = W + woff[p] + 3 * (size_t)k;  // [na][3]
            for (int c = 0; c < 3; ++c) w[c] = acc[c];
            for (int e = 0; e < 3; ++e)
                for (int c = 0; c < 3; ++c) {
                    double v = (double)zi[e] * acc[c];
                    if (a == b) {
                        const int i = members[abeg + k];
                        v += g.selfc * zq[3 * i + e] * zq[3 * i + c];
                    }
                    cacc[3 * e + c] += v;
                }
        }
    }
    block_sum<9>(cacc, red);
    if (threadIdx.x == 0) {
        if (Cblk) {  // sparse coarse operator: the pair's own 3 x 3 block
            for (int t = 0; t < 9; ++t) Cblk[9 * (size_t)p + t] = cacc[t];
        } else {
            for (int e = 0; e < 3; ++e)
                for (int c = 0; c < 3; ++c) C[(size_t)(3 * a + e) * ldc + 3 * b + c] += cacc[3 * e + c];
        }
    }
}

// Structure factors of the coarse columns: F[3a+e][2m] = sqrt(w_m) Re S_ae(k_m),
// F[3a+e][2m+1] = sqrt(w_m) Im S_ae(k_m).  One CTA per coarse body.
__global__ void coarse_wave_basis_kernel(int nmodes, const float4 *__restrict__ kv, const int *__restrict__ cbody,
                                         const int *__restrict__ body_start, const int *__restrict__ members,
                                         const double4 *__restrict__ pos, double3 Linv, const double *__restrict__ zq,
                                         int ldf, float *__restrict__ F) {
    __shared__ float4 sf[kChunk];
    __shared__ float2 sz[kChunk];
    const int a = blockIdx.x, ba = cbody[a];
    const int beg = body_start[ba], nb = body_start[ba + 1] - beg;
    for (int m0 = 0; m0 < nmodes; m0 += blockDim.x) {
        const int m = m0 + threadIdx.x;
        const float4 k = m < nmodes ? kv[m] : make_float4(0.f, 0.f, 0.f, 0.f);
        float re[3] = {0.f, 0.f, 0.f}, im[3] = {0.f, 0.f, 0.f};
        for (int j0 = 0; j0 < nb; j0 += kChunk) {
            const int nj = min(kChunk, nb - j0);
            __syncthreads();
            for (int t = threadIdx.x; t < nj; t += blockDim.x) {
                const int i = members[beg + j0 + t];
                const double4 p = pos[i];
                sf[t] = make_float4((float)(p.x * Linv.x), (float)(p.y * Linv.y), (float)(p.z * Linv.z),
                                    (float)zq[3 * i]);
                sz[t] = make_float2((float)zq[3 * i + 1], (float)zq[3 * i + 2]);
            }
            __syncthreads();
            if (m < nmodes) {
                for (int t = 0; t < nj; ++t) {
                    const float4 f = sf[t];
                    float s, c;
                    sincospif(2.0f * (k.x * f.x + k.y * f.y + k.z * f.z), &s, &c);
                    const float2 z12 = sz[t];
                    re[0] += f.w * c;
                    im[0] -= f.w * s;
                    re[1] += z12.x * c;
                    im[1] -= z12.x * s;
                    re[2] += z12.y * c;
                    im[2] -= z12.y * s;
                }
            }
        }
        if (m < nmodes)
            for (int e = 0; e < 3; ++e) {
                const int row = 3 * a + e;
                F[(size_t)row * ldf + 2 * m] = k.w * re[e];
                F[(size_t)row * ldf + 2 * m + 1] = k.w * im[e];
            }
    }
}

// C = F F^T (FP32 products, FP32 accumulation, written as FP64), n x n, K a multiple of 16.
__global__ void __launch_bounds__(256) syrk_kernel(int n, int K, const float *__restrict__ F, int ldf,
                                                   double *__restrict__ C, int ldc) {
    __shared__ float As[16][64 + 4], Bs[16][64 + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int r0 = blockIdx.y * 64, c0 = blockIdx.x * 64;
    float acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = 0.f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int t = threadIdx.x; t < 64 * 16; t += 256) {
            const int rr = t >> 4, kk = t & 15;
            As[kk][rr] = r0 + rr < n ? F[(size_t)(r0 + rr) * ldf + k0 + kk] : 0.f;
            Bs[kk][rr] = c0 + rr < n ? F[(size_t)(c0 + rr) * ldf + k0 + kk] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float av[4], bv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                av[u] = As[kk][ty * 4 + u];
                bv[u] = Bs[kk][tx * 4 + u];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] += av[u] * bv[v];
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int r = r0 + ty * 4 + u, c = c0 + tx * 4 + v;
            if (r < n && c < n) C[(size_t)r * ldc + c] = acc[u][v];
        }
}

// Padding rows/columns n..np of C: identity, so the inverse keeps them decoupled.
__global__ void pad_identity_kernel(int n, int np, double *__restrict__ C) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)np * np) return;
    const int r = (int)(t / np), c = (int)(t % np);
    if (r >= n || c >= n) C[t] = r == c ? 1.0 : 0.0;
}

// Symmetrise (the two orders of a near pair are summed separately) in place.
__global__ void symmetrise_kernel(int n, double *__restrict__ C, int ldc) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    const int r = (int)(t / n), c = (int)(t % n);
    if (c <= r) return;
    const double v = 0.5 * (C[(size_t)r * ldc + c] + C[(size_t)c * ldc + r]);
    C[(size_t)r * ldc + c] = v;
    C[(size_t)c * ldc + r] = v;
}

// ---- blocked Gauss-Jordan inversion of an SPD matrix, in place (no pivoting, FP32) ----
// Step k (block K = [k0, k0+NB)):  Dinv = A_KK^-1;  R = Dinv A_K* with A_KK := I;
// Fc = A_*K;  A_i* = (A_i* with A_iK := 0) - Fc_i R  (i not in K);  A_K* = R.
// FP32 is enough for a preconditioner: the coarse operators met here have condition
// numbers of 1e2-1e3, so C^-1 carries relative errors ~1e-4 at worst.
// Symmetry: with S the indices swept so far, A_ij = A_ji when i and j are both in S or both
// outside it, and A_ij = -A_ji otherwise (the sweep operator's sign rule); so only the
// 128 x 128 tiles on and below the diagonal are updated, the panels read the missing
// entries through that rule, and the upper tiles are mirrored at the end.

// Dinv of the pivot block (one CTA of kPivThreads threads, scalar in-place Gauss-Jordan in
// shared memory; thread t owns entries (t/64 + kPivStride u, t%64)); a pivot that is not
// positive and finite sets *flag and leaves Dinv untouched.
constexpr int kPivThreads = 256, kPivStride = kPivThreads / NB, kPivRows = NB / kPivStride;
__global__ void __launch_bounds__(kPivThreads) gj_pivot_kernel(int k0, int np, const float *__restrict__ A,
                                                               float *__restrict__ Dinv, int *__restrict__ flag) {
    __shared__ float D[NB][NB + 1];
    const int c = threadIdx.x % NB, r0 = threadIdx.x / NB;
#pragma unroll
    for (int u = 0; u < kPivRows; ++u)
        D[r0 + kPivStride * u][c] = A[(size_t)(k0 + r0 + kPivStride * u) * np + k0 + c];
    __syncthreads();
    for (int s = 0; s < NB; ++s) {
        const float piv = D[s][s];
        if (!(piv > 0.0f) || !isfinite(piv)) {  // uniform over the block
            if (threadIdx.x == 0) atomicExch(flag, 1);
            return;
        }
        const float inv = 1.0f / piv;
        float rs[kPivRows];
#pragma unroll
        for (int u = 0; u < kPivRows; ++u) rs[u] = D[r0 + kPivStride * u][s];
        const float sc = D[s][c];
        __syncthreads();
        // row s: scaled, with the identity column in place of column s;
        // other rows: D[r][c] -= D[r][s] D[s][c] / piv, and column s becomes -D[r][s] / piv
        const float scs = c == s ? inv : sc * inv;
#pragma unroll
        for (int u = 0; u < kPivRows; ++u) {
            const int r = r0 + kPivStride * u;
            if (r == s) D[r][c] = scs;
            else D[r][c] = c == s ? -rs[u] * inv : D[r][c] - rs[u] * scs;
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < kPivRows; ++u) Dinv[(r0 + kPivStride * u) * NB + c] = D[r0 + kPivStride * u][c];
}

// R = Dinv A_K* (with A_KK := I, so R_KK = Dinv) and Fc = A_*K.  blockIdx.x: 64 columns.
__global__ void gj_panel_kernel(int k0, int np, const float *__restrict__ A, const float *__restrict__ Dinv,
                                float *__restrict__ R, float *__restrict__ Fc) {
    __shared__ float Ds[NB][NB + 1];
    __shared__ float As[NB][NB + 1];
    const int j0 = blockIdx.x * NB;
    const int tK = k0 / GT, tj = j0 / GT;
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        const int r = t / NB, c = t % NB;
        Ds[r][c] = Dinv[t];
        // A_K,j right of the pivot's tile: from the stored A_j,K (both unswept: same sign)
        As[r][c] = tj > tK ? A[(size_t)(j0 + c) * np + k0 + r] : A[(size_t)(k0 + r) * np + j0 + c];
    }
    __syncthreads();
    const bool diag = j0 == k0;
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        const int r = t / NB, c = t % NB;
        float v;
        if (diag) {
            v = Ds[r][c];
        } else {
            v = 0.0f;
#pragma unroll 16
            for (int s = 0; s < NB; ++s) v += Ds[r][s] * As[s][c];
        }
        R[(size_t)r * np + j0 + c] = v;
    }
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {  // rows j0.. of the column panel
        const int r = t / NB, c = t % NB;
        // A_i,K above the pivot's tile: i swept, K not, so A_i,K = -A_K,i
        Fc[(size_t)(j0 + r) * NB + c] =
            tj < tK ? -A[(size_t)(k0 + c) * np + j0 + r] : A[(size_t)(j0 + r) * np + k0 + c];
    }
}

// A_i* = (A_i*, A_iK := 0) - Fc_i R for i outside K; A_K* = R.  128 x 128 tile per CTA,
// 8 x 8 outputs per thread (rows and columns {4t..4t+3} and {64+4t..64+4t+3}, so every
// shared-memory read is a conflict-free float4), the inner dimension in two halves of 32.
__global__ void __launch_bounds__(256) gj_update_kernel(int k0, int np, float *__restrict__ A,
                                                        const float *__restrict__ R, const float *__restrict__ Fc) {
    __shared__ __align__(16) float Fs[32][GT + 4];
    __shared__ __align__(16) float Rs[32][GT + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    // block b -> lower tile (tr, tc), tc <= tr, b = tr (tr + 1) / 2 + tc
    int tr = (int)((sqrtf(8.0f * blockIdx.x + 1.0f) - 1.0f) * 0.5f);
    while ((tr + 1) * (tr + 2) / 2 <= (int)blockIdx.x) ++tr;
    while (tr * (tr + 1) / 2 > (int)blockIdx.x) --tr;
    const int tc = blockIdx.x - tr * (tr + 1) / 2;
    const int r0 = tr * GT, c0 = tc * GT;
    float acc[8][8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = 0.f;
    for (int s0 = 0; s0 < NB; s0 += 32) {
        for (int f = threadIdx.x; f < GT * 8; f += 256) {
            const int q = f % GT, j = f / GT;  // row r0+q of the column panel, entries s0+4j..
            const float4 v = *reinterpret_cast<const float4 *>(Fc + (size_t)(r0 + q) * NB + s0 + 4 * j);
            Fs[4 * j][q] = v.x;
            Fs[4 * j + 1][q] = v.y;
            Fs[4 * j + 2][q] = v.z;
            Fs[4 * j + 3][q] = v.w;
            const int sr = f / 32, c4 = f % 32;
            *reinterpret_cast<float4 *>(&Rs[sr][4 * c4]) =
                *reinterpret_cast<const float4 *>(R + (size_t)(s0 + sr) * np + c0 + 4 * c4);
        }
        __syncthreads();
#pragma unroll 4
        for (int s = 0; s < 32; ++s) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&Fs[s][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&Fs[s][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&Rs[s][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&Rs[s][64 + tx * 4]);
            const float fa[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float fb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int v = 0; v < 8; ++v) acc[u][v] += fa[u] * fb[v];
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int i = r0 + (u < 4 ? ty * 4 + u : 64 + ty * 4 + u - 4);
        const bool krow = i >= k0 && i < k0 + NB;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = c0 + h * 64 + tx * 4;
            float4 *dst = reinterpret_cast<float4 *>(A + (size_t)i * np + j);
            if (krow) {  // the pivot rows take R
                *dst = *reinterpret_cast<const float4 *>(R + (size_t)(i - k0) * np + j);
            } else {
                const bool kcol = j >= k0 && j < k0 + NB;
                const float4 old = kcol ? make_float4(0.f, 0.f, 0.f, 0.f) : *dst;
                *dst = make_float4(old.x - acc[u][4 * h], old.y - acc[u][4 * h + 1], old.z - acc[u][4 * h + 2],
                                   old.w - acc[u][4 * h + 3]);
            }
        }
    }
}

// The upper tiles from the lower ones (the inverse is symmetric).
__global__ void mirror_upper_kernel(int np, float *__restrict__ A) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)np * np) return;
    const int r = (int)(t / np), c = (int)(t % np);
    if (r / GT < c / GT) A[t] = A[(size_t)c * np + r];
}

__global__ void to_float_kernel(long long n, const double *__restrict__ a, float *__restrict__ b) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) b[t] = (float)a[t];
}

// sum_c row[c] v[c] over a zero-padded row of n4 float4 (one warp; row 16-byte aligned).
__device__ __forceinline__ double warp_row_dot(const float *__restrict__ row, const double *__restrict__ v, int n4) {
    const int lane = threadIdx.x & 31;
    const float4 *r4 = reinterpret_cast<const float4 *>(row);
    const double2 *v2 = reinterpret_cast<const double2 *>(v);
    double s0 = 0.0, s1 = 0.0;
#pragma unroll 4
    for (int c = lane; c < n4; c += 32) {
        const float4 a = __ldg(r4 + c);
        const double2 p = v2[2 * c], q = v2[2 * c + 1];
        s0 += (double)a.x * p.x + (double)a.y * p.y;
        s1 += (double)a.z * q.x + (double)a.w * q.y;
    }
    double s = s0 + s1;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// ---- sparse coarse level: block-Jacobi preconditioned CG ----
// For coarse problems above the dense limit the coarse operator is kept as 3 x 3 blocks of
// the near pairs (self and real-space terms) plus the low-rank wave-space term F F^T, and
// C y = -g is solved approximately by a fixed number of conjugate-gradient steps with the
// inverse diagonal blocks as preconditioner; the flexible outer iteration accepts the
// resulting (slightly varying) preconditioner.  Sums over blocks are reduced in a fixed
// order.
constexpr int kVecThreads = 256, kSpmvWarpsC = 8;

// sum of a[0..n) on every thread of the block (fixed order: strided partial sums, tree)
__device__ double block_sum_array(const double *__restrict__ a, int n, double *red /* [32] */) {
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += a[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += red[w];
    __syncthreads();
    return t;
}

__device__ __forceinline__ void mat3_vec(const double *__restrict__ M, const double v[3], double out[3]) {
    for (int e = 0; e < 3; ++e) out[e] = M[3 * e] * v[0] + M[3 * e + 1] * v[1] + M[3 * e + 2] * v[2];
}

// inverse of each body's diagonal block (symmetrised); a block that is not positive
// definite sets *flag
__global__ void block_jacobi_kernel(int nbc, const int *__restrict__ phead, const int *__restrict__ pcount,
                                    const int *__restrict__ pair_b, const double *__restrict__ Cblk,
                                    const float *__restrict__ F, int K2, double *__restrict__ Dblk,
                                    int *__restrict__ flag) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nbc) return;
    int q = -1;
    for (int k = 0; k < pcount[a]; ++k)
        if (pair_b[phead[a] + k] == a) q = phead[a] + k;
    double m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (q >= 0)
        for (int e = 0; e < 3; ++e)
            for (int c = 0; c < 3; ++c) m[3 * e + c] = 0.5 * (Cblk[9 * (size_t)q + 3 * e + c] + Cblk[9 * (size_t)q + 3 * c + e]);
    for (int e = 0; e < 3; ++e)  // + the wave-space part F_a F_a^T
        for (int c = 0; c < 3; ++c) {
            const float *fe = F + (size_t)(3 * a + e) * K2, *fc = F + (size_t)(3 * a + c) * K2;
            double t = 0.0;
            for (int k = 0; k < K2; ++k) t += (double)fe[k] * fc[k];
            m[3 * e + c] += t;
        }
    const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    double *d = Dblk + 9 * (size_t)a;
    if (!(det > 0.0) || !(m[0] > 0.0) || !isfinite(det)) {
        atomicExch(flag, 1);
        for (int t = 0; t < 9; ++t) d[t] = 0.0;
        return;
    }
    const double id = 1.0 / det;
    d[0] = c00 * id;
    d[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    d[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    d[3] = c01 * id;
    d[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    d[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    d[6] = c02 * id;
    d[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    d[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

// u = F^T v in two steps: partial column sums over chunks of kColRows rows of F (threads
// over the columns, every load coalesced), then a reduction over the chunks in a fixed
// order.  With kv, u[k] is also scaled by sqrt(w) of its wave vector (k / 2).  Chunks of 8
// rows give ~375 CTAs for 3000 coarse unknowns (32-row chunks left most SMs idle).
constexpr int kColRows = 8;
__device__ __forceinline__ void fcol_partial_chunk(int chunk, int nc, int K2, const float *__restrict__ F,
                                                   const double *__restrict__ v, double *__restrict__ part) {
    const int c0 = chunk * kColRows, c1 = min(nc, c0 + kColRows);
    for (int k = threadIdx.x; k < K2; k += blockDim.x) {
        double acc = 0.0;
#pragma unroll 8
        for (int c = c0; c < c1; ++c) acc += (double)__ldg(F + (size_t)c * K2 + k) * v[c];
        part[(size_t)chunk * K2 + k] = acc;
    }
}

__global__ void __launch_bounds__(256) fcol_partial_kernel(int nc, int K2, const float *__restrict__ F,
                                                           const double *__restrict__ v, double *__restrict__ part) {
    fcol_partial_chunk(blockIdx.x, nc, K2, F, v, part);
}

template <typename T>
__device__ __forceinline__ void fcol_reduce_block(int blk, int nchunk, int K2, const double *__restrict__ part,
                                                  int nmodes, const float4 *__restrict__ kv, T *__restrict__ u) {
    // one warp per column: lane l sums chunks l, l+32, ..., then a fixed shuffle tree
    const int k = (blk * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (k >= K2) return;
    double s = 0.0;
    for (int q = lane; q < nchunk; q += 32) s += part[(size_t)q * K2 + k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane != 0) return;
    if (kv) s = k < 2 * nmodes ? s * kv[k >> 1].w : 0.0;
    u[k] = (T)s;
}

template <typename T>
__global__ void fcol_reduce_kernel(int nchunk, int K2, const double *__restrict__ part, int nmodes,
                                   const float4 *__restrict__ kv, T *__restrict__ u) {
    fcol_reduce_block<T>(blockIdx.x, nchunk, K2, part, nmodes, kv, u);
}

// y = 0, r = -g, z = D r, p = z; partial r.z per block
__global__ void __launch_bounds__(kVecThreads) pcg_init_kernel(int nbc, const double *__restrict__ Dblk,
                                                               const double *__restrict__ g, double *__restrict__ y,
                                                               double *__restrict__ r, double *__restrict__ z,
                                                               double *__restrict__ p, double *__restrict__ part_rz) {
    __shared__ double red[32];
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    double rz = 0.0;
    if (a < nbc) {
        const double rv[3] = {-g[3 * a], -g[3 * a + 1], -g[3 * a + 2]};
        double zv[3];
        mat3_vec(Dblk + 9 * (size_t)a, rv, zv);
        for (int e = 0; e < 3; ++e) {
            y[3 * a + e] = 0.0;
            r[3 * a + e] = rv[e];
            z[3 * a + e] = zv[e];
            p[3 * a + e] = zv[e];
            rz += rv[e] * zv[e];
        }
    }
    double v[1] = {rz};
    block_sum<1>(v, red);
    if (threadIdx.x == 0) part_rz[blockIdx.x] = v[0];
}

// q = C p (one warp per body, lanes over its near pairs); partial p.q per block
__global__ void __launch_bounds__(kSpmvWarpsC * 32) pcg_spmv_kernel(int nbc, const int *__restrict__ phead,
                                                                    const int *__restrict__ pcount,
                                                                    const int *__restrict__ pair_b,
                                                                    const double *__restrict__ Cblk,
                                                                    const float *__restrict__ F, int K2,
                                                                    const double *__restrict__ u,
                                                                    const double *__restrict__ p,
                                                                    double *__restrict__ q,
                                                                    double *__restrict__ part_pq) {
    __shared__ double red[32];
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    double pq = 0.0;
    if (a < nbc) {
        double acc[3] = {0.0, 0.0, 0.0};
        const int h0 = phead[a], n = pcount[a];
        for (int k = lane; k < n; k += 32) {
            const int b = pair_b[h0 + k];
            const double pb[3] = {p[3 * b], p[3 * b + 1], p[3 * b + 2]};
            double t[3];
            mat3_vec(Cblk + 9 * (size_t)(h0 + k), pb, t);
            for (int e = 0; e < 3; ++e) acc[e] += t[e];
        }
        for (int k = lane; k < K2; k += 32) {  // + (F F^T p)_a = F_a u
            const double uk = u[k];
            for (int e = 0; e < 3; ++e) acc[e] += (double)F[(size_t)(3 * a + e) * K2 + k] * uk;
        }
        for (int e = 0; e < 3; ++e)
            for (int o = 16; o > 0; o >>= 1) acc[e] += __shfl_xor_sync(0xffffffffu, acc[e], o);
        if (lane == 0) {
            for (int e = 0; e < 3; ++e) q[3 * a + e] = acc[e];
            pq = p[3 * a] * acc[0] + p[3 * a + 1] * acc[1] + p[3 * a + 2] * acc[2];
        }
    }
    double v[1] = {pq};
    block_sum<1>(v, red);
    if (threadIdx.x == 0) part_pq[blockIdx.x] = v[0];
}

// alpha = (r.z) / (p.q); y += alpha p; r -= alpha q; z = D r; partial r.z (new) per block
__global__ void __launch_bounds__(kVecThreads) pcg_update_kernel(int nbc, int nspmv, const double *__restrict__ part_pq,
                                                                 int nvec, const double *__restrict__ part_rz,
                                                                 const double *__restrict__ Dblk,
                                                                 const double *__restrict__ p,
                                                                 const double *__restrict__ q,
                                                                 double *__restrict__ y, double *__restrict__ r,
                                                                 double *__restrict__ z,
                                                                 double *__restrict__ part_rz_next) {
    __shared__ double red[32];
    const double pq = block_sum_array(part_pq, nspmv, red);
    const double rz = block_sum_array(part_rz, nvec, red);
    const double alpha = pq > 0.0 ? rz / pq : 0.0;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    double rzn = 0.0;
    if (a < nbc) {
        double rv[3];
        for (int e = 0; e < 3; ++e) {
            y[3 * a + e] += alpha * p[3 * a + e];
            rv[e] = r[3 * a + e] - alpha * q[3 * a + e];
            r[3 * a + e] = rv[e];
        }
        double zv[3];
        mat3_vec(Dblk + 9 * (size_t)a, rv, zv);
        for (int e = 0; e < 3; ++e) {
            z[3 * a + e] = zv[e];
            rzn += rv[e] * zv[e];
        }
    }
    double v[1] = {rzn};
    block_sum<1>(v, red);
    if (threadIdx.x == 0) part_rz_next[blockIdx.x] = v[0];
}

// p = z + beta p, beta = (r.z)_new / (r.z)_old
__global__ void __launch_bounds__(kVecThreads) pcg_dir_kernel(int nbc, int nvec, const double *__restrict__ part_old,
                                                              const double *__restrict__ part_new,
                                                              const double *__restrict__ z, double *__restrict__ p) {
    __shared__ double red[32];
    const double ro = block_sum_array(part_old, nvec, red);
    const double rn = block_sum_array(part_new, nvec, red);
    const double beta = ro > 0.0 ? rn / ro : 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 3 * nbc) p[i] = z[i] + beta * p[i];
}

// ---- application ----

// g[3a+e] = sum_{i in a} z_ae(i) x_i + zp[a][e] x[N+a]
__device__ __forceinline__ void coarse_restrict_body(int a, int N, const int *__restrict__ cbody,
                                                     const int *__restrict__ body_start,
                                                     const int *__restrict__ members, const double *__restrict__ zq,
                                                     const double *__restrict__ zp, const double *__restrict__ x,
                                                     double *__restrict__ g) {
    __shared__ double red[3 * 32];
    const int ba = cbody[a];
    const int beg = body_start[ba], nb = body_start[ba + 1] - beg;
    double s[3] = {0.0, 0.0, 0.0};
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        const int i = members[beg + k];
        const double xi = x[i];
        for (int e = 0; e < 3; ++e) s[e] += zq[3 * i + e] * xi;
    }
    block_sum<3>(s, red);
    if (threadIdx.x == 0)
        for (int e = 0; e < 3; ++e) g[3 * a + e] = s[e] + zp[3 * ba + e] * x[N + ba];
}

__global__ void coarse_restrict_kernel(int N, const int *__restrict__ cbody, const int *__restrict__ body_start,
                                       const int *__restrict__ members, const double *__restrict__ zq,
                                       const double *__restrict__ zp, const double *__restrict__ x,
                                       double *__restrict__ g) {
    coarse_restrict_body(blockIdx.x, N, cbody, body_start, members, zq, zp, x, g);
}

// y = -Cinv g (one warp per row; rows of ld floats, g zero beyond n)
__device__ __forceinline__ void coarse_gemv_block(int blk, int n, int ld, const float *__restrict__ Ci,
                                                  const double *__restrict__ g, double *__restrict__ y) {
    const int r = (blk * blockDim.x + threadIdx.x) >> 5;
    if (r >= n) return;
    const double s = warp_row_dot(Ci + (size_t)r * ld, g, ld / 4);
    if ((threadIdx.x & 31) == 0) y[r] = -s;
}

__global__ void coarse_gemv_kernel(int n, int ld, const float *__restrict__ Ci, const double *__restrict__ g,
                                   double *__restrict__ y) {
    coarse_gemv_block(blockIdx.x, n, ld, Ci, g, y);
}

// sin and cos of 2 pi t: t reduced to [-1/2, 1/2] first, then the fast intrinsic, whose
// absolute error on [-pi, pi] is below 4e-7
__device__ __forceinline__ void sincos_turns(float t, float *s, float *c) {
    __sincosf(6.283185307179586f * (t - rintf(t)), s, c);
}

// t = x - A~ Z y on the bead rows of body b (one CTA per body), t[N+b] = x[N+b]:
//   (A~ Z y)_i = Phi_b(Z y) - [ self (Z_q y)_i + sum_p W_p y_b(p) + wave_i ],
//   wave_i = sum_m (cos(k_m.r_i) u_re[m] - sin(k_m.r_i) u_im[m]).
// The wave vectors come in rows of consecutive m_z at fixed (m_x, m_y): one sine/cosine per
// row, then rotation by exp(2 pi i z / L_z) along the row.  The body's near pairs (partner
// coefficients and W offsets) are staged in shared memory first.
__device__ __forceinline__ void coarse_model_body(int b, int N, int nmodes, int nrows, const int4 *__restrict__ rows,
                                                  const int *__restrict__ cidx, const int *__restrict__ body_start,
                                                  const int *__restrict__ members, const double4 *__restrict__ pos,
                                                  double3 Linv, const double *__restrict__ zq,
                                                  const double *__restrict__ zp, const int *__restrict__ phead,
                                                  const int *__restrict__ pcount, const int *__restrict__ pair_b,
                                                  const long long *__restrict__ woff, const float *__restrict__ W,
                                                  const float *__restrict__ u, double selfc,
                                                  const double *__restrict__ y, const double *__restrict__ x,
                                                  double *__restrict__ t, int split) {
    extern __shared__ float4 dyn[];
    const int beg = body_start[b], nb = body_start[b + 1] - beg;
    const int a = cidx[b];
    const int h0 = a >= 0 ? phead[a] : 0, npr = a >= 0 ? pcount[a] : 0;
    int4 *srow = reinterpret_cast<int4 *>(dyn);                                // [nrows] (mx, my, mz0, first mode)
    float2 *su = reinterpret_cast<float2 *>(dyn + nrows);                     // [nmodes]
    double2 *sy = reinterpret_cast<double2 *>(dyn + nrows + (nmodes + 1) / 2); // [npr][2] partner y, W offset
    double *red = reinterpret_cast<double *>(sy + 2 * npr);                    // [split-1][P] partial sums
    for (int q = threadIdx.x; q < nrows; q += blockDim.x) srow[q] = rows[q];
    for (int q = threadIdx.x; q < nmodes; q += blockDim.x) su[q] = make_float2(u[2 * q], u[2 * q + 1]);
    for (int q = threadIdx.x; q < npr; q += blockDim.x) {
        const int c = pair_b[h0 + q];
        sy[2 * q] = make_double2(y[3 * c], y[3 * c + 1]);
        sy[2 * q + 1] = make_double2(y[3 * c + 2], __longlong_as_double(woff[h0 + q]));
    }
    __syncthreads();
    // `split` threads per bead (P = blockDim / split >= the body's beads when split > 1):
    // part s takes the near pairs and the wave rows q = s, s + split, ...; the parts'
    // sums meet in shared memory
    const int P = blockDim.x / split, part = threadIdx.x / P, k0 = threadIdx.x % P;
    for (int k = k0; k < nb || (split > 1 && k == k0); k += P) {
        const bool mine = k < nb;
        const int i = mine ? members[beg + k] : 0;
        double m0 = 0.0, m1 = 0.0;
#pragma unroll 4
        for (int q = part; q < (mine ? npr : 0); q += split) {
            const double2 y01 = sy[2 * q], y2o = sy[2 * q + 1];
            const float *w = W + __double_as_longlong(y2o.y) + 3 * (size_t)k;
            const float w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2);
            m0 += (double)w0 * y01.x + (double)w1 * y01.y;
            m1 += (double)w2 * y2o.x;
        }
        const double4 p = mine ? pos[i] : make_double4(0, 0, 0, 0);
        const float fx = (float)(p.x * Linv.x), fy = (float)(p.y * Linv.y), fz = (float)(p.z * Linv.z);
        float sz, cz;
        sincos_turns(fz, &sz, &cz);
        float wave = 0.f;
        for (int q = part; q < (mine ? nrows : 0); q += split) {
            const int4 r = srow[q];
            const int end = q + 1 < nrows ? srow[q + 1].w : nmodes;
            float s, c;
            sincos_turns((float)r.x * fx + (float)r.y * fy + (float)r.z * fz, &s, &c);
            for (int mm = r.w; mm < end; ++mm) {
                const float2 uu = su[mm];
                wave += c * uu.x - s * uu.y;
                const float c2 = c * cz - s * sz;
                s = s * cz + c * sz;
                c = c2;
            }
        }
        double m = (double)wave + m0 + m1;
        if (split > 1) {
            if (part > 0 && mine) red[(part - 1) * P + k] = m;
            __syncthreads();
            if (part > 0 || !mine) continue;
            for (int v = 1; v < split; ++v) m += red[(v - 1) * P + k];
        }
        double phi = 0.0;
        if (a >= 0) {
            const double y0 = y[3 * a], y1 = y[3 * a + 1], y2 = y[3 * a + 2];
            m += selfc * (zq[3 * i] * y0 + zq[3 * i + 1] * y1 + zq[3 * i + 2] * y2);
            phi = zp[3 * b] * y0 + zp[3 * b + 1] * y1 + zp[3 * b + 2] * y2;
        }
        t[i] = x[i] - (phi - m);
    }
    if (threadIdx.x == 0) t[N + b] = x[N + b];
}

__global__ void coarse_model_kernel(int N, int nmodes, int nrows, const int4 *__restrict__ rows,
                                    const int *__restrict__ cidx, const int *__restrict__ body_start,
                                    const int *__restrict__ members, const double4 *__restrict__ pos, double3 Linv,
                                    const double *__restrict__ zq, const double *__restrict__ zp,
                                    const int *__restrict__ phead, const int *__restrict__ pcount,
                                    const int *__restrict__ pair_b, const long long *__restrict__ woff,
                                    const float *__restrict__ W, const float *__restrict__ u, double selfc,
                                    const double *__restrict__ y, const double *__restrict__ x,
                                    double *__restrict__ t, int split) {
    coarse_model_body(blockIdx.x, N, nmodes, nrows, rows, cidx, body_start, members, pos, Linv, zq, zp, phead, pcount,
                      pair_b, woff, W, u, selfc, y, x, t, split);
}

// z += Z y
__device__ __forceinline__ void coarse_prolong_body(int a, int N, const int *__restrict__ cbody,
                                                    const int *__restrict__ body_start,
                                                    const int *__restrict__ members, const double *__restrict__ zq,
                                                    const double *__restrict__ zp, const double *__restrict__ y,
                                                    double *__restrict__ z) {
    const int ba = cbody[a];
    const int beg = body_start[ba], nb = body_start[ba + 1] - beg;
    const double y0 = y[3 * a], y1 = y[3 * a + 1], y2 = y[3 * a + 2];
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        const int i = members[beg + k];
        z[i] += zq[3 * i] * y0 + zq[3 * i + 1] * y1 + zq[3 * i + 2] * y2;
    }
    if (threadIdx.x == 0) z[N + ba] += zp[3 * ba] * y0 + zp[3 * ba + 1] * y1 + zp[3 * ba + 2] * y2;
}

__global__ void coarse_prolong_kernel(int N, const int *__restrict__ cbody, const int *__restrict__ body_start,
                                      const int *__restrict__ members, const double *__restrict__ zq,
                                      const double *__restrict__ zp, const double *__restrict__ y,
                                      double *__restrict__ z) {
    coarse_prolong_body(blockIdx.x, N, cbody, body_start, members, zq, zp, y, z);
}

// ---- lockstep batches: the same bodies, one CTA per (replica, item) of the replicas
// whose coarse level is active ----
__global__ void restrict_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                      const int *__restrict__ mask, int xin) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &r = reps[it.x];
    if (!r.coarse) return;
    coarse_restrict_body(it.y, r.N, r.cbody, r.body_start, r.body_members, r.zq, r.zpv, r.vec[xin], r.cg);
}

__global__ void gemv_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                  const int *__restrict__ mask) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &r = reps[it.x];
    if (!r.coarse) return;
    coarse_gemv_block(it.y, r.nc, r.np, r.Ci, r.cg, r.cy);
}

__global__ void __launch_bounds__(256) fpart_batch_kernel(const BatchRep *__restrict__ reps,
                                                          const int2 *__restrict__ items,
                                                          const int *__restrict__ mask) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &r = reps[it.x];
    if (!r.coarse || r.nmodes == 0) return;
    fcol_partial_chunk(it.y, r.nc, r.K2, r.F, r.cy, r.fpart);
}

__global__ void freduce_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                     const int *__restrict__ mask) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &r = reps[it.x];
    if (!r.coarse || r.nmodes == 0) return;
    fcol_reduce_block<float>(it.y, (r.nc + kColRows - 1) / kColRows, r.K2, r.fpart, r.nmodes, r.kv, r.cu);
}

__global__ void __launch_bounds__(128, 10) model_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                   const int *__restrict__ mask, int xin, int split) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &r = reps[it.x];
    if (!r.coarse) return;
    coarse_model_body(it.y, r.N, r.nmodes, r.nrows, r.rows, r.cidx, r.body_start, r.body_members, r.pos64,
                      make_double3(r.Linv[0], r.Linv[1], r.Linv[2]), r.zq, r.zpv, r.phead, r.pcount, r.pair_b, r.woff,
                      r.W, r.cu, r.selfc, r.cy, r.vec[xin], r.ct, split);
}

__global__ void prolong_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                     const int *__restrict__ mask, int zout) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &r = reps[it.x];
    if (!r.coarse) return;
    coarse_prolong_body(it.y, r.N, r.cbody, r.body_start, r.body_members, r.zq, r.zpv, r.cy, r.vec[zout]);
}

template <typename T> int grow(cr_handle *h, T **p, size_t &cap, size_t need, bool &moved) {
    if (need <= cap && *p) return CR_OK;
    CR_TRY(dalloc(h, p, std::max<size_t>(need, 1)));
    cap = std::max<size_t>(need, 1);
    moved = true;
    return CR_OK;
}

}  // namespace

void coarse_free(cr_handle *h) {
    CoarseSpace &c = h->coarse;
    dfree(&c.cidx);
    dfree(&c.cbody);
    dfree(&c.zq);
    dfree(&c.zp);
    dfree(&c.cent);
    dfree(&c.basis);
    dfree(&c.phead);
    dfree(&c.pcount);
    dfree(&c.pair_a);
    dfree(&c.pair_b);
    dfree(&c.woff);
    dfree(&c.W);
    dfree(&c.kv);
    dfree(&c.rows);
    dfree(&c.Cblk);
    dfree(&c.Dblk);
    dfree(&c.pr);
    dfree(&c.pz);
    dfree(&c.pp);
    dfree(&c.pq);
    dfree(&c.part_pq);
    dfree(&c.part_rz);
    dfree(&c.pu);
    dfree(&c.F);
    dfree(&c.fpart);
    dfree(&c.C);
    dfree(&c.Ci);
    dfree(&c.R);
    dfree(&c.Fc);
    dfree(&c.Dinv);
    dfree(&c.g);
    dfree(&c.y);
    dfree(&c.u);
    dfree(&c.t);
    const int max_dense = c.max_dense, pcg_iters = c.pcg_iters;  // caller settings survive
    c = CoarseSpace{};
    c.max_dense = max_dense;
    c.pcg_iters = pcg_iters;
}

int coarse_prepare(cr_handle *h) {
    CoarseSpace &cs = h->coarse;
    if (h->user.precond != CR_PRECOND_TWO_LEVEL) return CR_OK;
    if (cs.gen == h->geo_gen) return CR_OK;
    ProfScope ps(h, PROF_COARSE);
    if (!h->cond.ready) CR_TRY(conductor_setup(h));
    const int N = h->N, B = h->B;
    cs.active = false;
    cs.nbc = 0;
    cs.nc = 0;
    cs.failed = false;
    // coarse bodies: rigid, at least kMinBeads beads
    std::vector<uint8_t> rigid(B);
    if (B > 0)
        CR_CUDA(h, cudaMemcpyAsync(rigid.data(), h->d_rigid, B, cudaMemcpyDeviceToHost, h->stream));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    std::vector<int> cidx(B, -1), cbody;
    for (int b = 0; b < B; ++b)
        if (rigid[b] && h->h_body_start[b + 1] - h->h_body_start[b] >= kMinBeads) {
            cidx[b] = (int)cbody.size();
            cbody.push_back(b);
        }
    const int nbc = (int)cbody.size(), nc = 3 * nbc;
    const bool sparse = nc > cs.max_dense;  // above the dense limit: near-pair blocks and PCG
    if (nbc == 0 || nc > kMaxSparse || (sparse && cs.pcg_iters == 0)) {
        cs.gen = h->geo_gen;
        return CR_OK;
    }
    bool moved = false;
    const size_t n1 = (size_t)N + B;
    CR_TRY(grow(h, &cs.cidx, cs.cap_cidx, (size_t)B, moved));
    CR_TRY(grow(h, &cs.cbody, cs.cap_cbody, (size_t)nbc, moved));
    CR_TRY(grow(h, &cs.zq, cs.cap_zq, 3 * (size_t)N, moved));
    CR_TRY(grow(h, &cs.zp, cs.cap_zp, 3 * (size_t)B, moved));
    CR_TRY(grow(h, &cs.cent, cs.cap_cent, (size_t)B, moved));
    CR_TRY(grow(h, &cs.basis, cs.cap_basis, 6 * n1, moved));
    CR_TRY(grow(h, &cs.phead, cs.cap_phead, (size_t)nbc, moved));
    CR_TRY(grow(h, &cs.pcount, cs.cap_pcount, (size_t)nbc, moved));
    CR_CUDA(h, cudaMemcpyAsync(cs.cidx, cidx.data(), B * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CR_CUDA(h, cudaMemcpyAsync(cs.cbody, cbody.data(), nbc * sizeof(int), cudaMemcpyHostToDevice, h->stream));

    const double3 L = make_double3(h->L[0], h->L[1], h->L[2]);
    const double3 Linv = make_double3(1.0 / h->L[0], 1.0 / h->L[1], 1.0 / h->L[2]);
    // basis: three conductor solves
    basis_rhs_kernel<<<blocks_for((long)n1, 256), 256, 0, h->stream>>>(N, B, h->d_body, h->d_body_start,
                                                                        h->d_body_members, h->m64.pos, L, Linv,
                                                                        cs.basis);
    CR_LAUNCH(h, "basis_rhs_kernel");
    for (int e = 0; e < 3; ++e) CR_TRY(conductor_apply(h, cs.basis + e * n1, cs.basis + (3 + e) * n1));
    basis_pack_kernel<<<B, 128, 0, h->stream>>>(N, B, h->d_body_start, h->d_body_members, cs.cidx, h->m64.pos, L,
                                                Linv, cs.basis + 3 * n1, cs.zq, cs.zp, cs.cent);
    CR_LAUNCH(h, "basis_pack_kernel");

    // near body pairs
    const double rc = h->d.rcut;
    near_pairs_kernel<false><<<blocks_for((long)nbc * 32, 256), 256, 0, h->stream>>>(
        nbc, cs.cbody, cs.cent, L, Linv, rc, cs.pcount, nullptr, nullptr);
    CR_LAUNCH(h, "near_pairs_kernel");
    std::vector<int> pcount(nbc), phead(nbc);
    std::vector<double4> cent(B);
    CR_CUDA(h, cudaMemcpyAsync(pcount.data(), cs.pcount, nbc * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CR_CUDA(h, cudaMemcpyAsync(cent.data(), cs.cent, B * sizeof(double4), cudaMemcpyDeviceToHost, h->stream));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    long long npairs = 0, wtotal = 0;
    std::vector<long long> woff;
    std::vector<int> pair_a;
    for (int a = 0; a < nbc; ++a) {
        phead[a] = (int)npairs;
        const int na = h->h_body_start[cbody[a] + 1] - h->h_body_start[cbody[a]];
        for (int q = 0; q < pcount[a]; ++q) {
            woff.push_back(wtotal);
            pair_a.push_back(a);
            wtotal += 3LL * na;
        }
        npairs += pcount[a];
    }
    if (npairs > INT32_MAX) return fail(h, CR_BAD_PARAM, "coarse level: too many near body pairs");
    CR_TRY(grow(h, &cs.pair_a, cs.cap_pair_a, (size_t)npairs, moved));
    CR_TRY(grow(h, &cs.pair_b, cs.cap_pair_b, (size_t)npairs, moved));
    CR_TRY(grow(h, &cs.woff, cs.cap_woff, (size_t)npairs, moved));
    CR_TRY(grow(h, &cs.W, cs.cap_W, (size_t)wtotal, moved));
    CR_CUDA(h, cudaMemcpyAsync(cs.phead, phead.data(), nbc * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CR_CUDA(h, cudaMemcpyAsync(cs.pair_a, pair_a.data(), npairs * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CR_CUDA(h, cudaMemcpyAsync(cs.woff, woff.data(), npairs * sizeof(long long), cudaMemcpyHostToDevice, h->stream));
    near_pairs_kernel<true><<<blocks_for((long)nbc * 32, 256), 256, 0, h->stream>>>(
        nbc, cs.cbody, cs.cent, L, Linv, rc, nullptr, cs.phead, cs.pair_b);
    CR_LAUNCH(h, "near_pairs_kernel");

    // wave vectors of the half space with 0 < |k| < kc (kc lowered if there are too many)
    const double xi = h->user.xi, V = h->L[0] * h->L[1] * h->L[2];
    double kc = 2.0 * xi;
    const int max_modes = sparse ? kMaxModesSparse : kMaxModes;
    std::vector<float4> kv;
    for (int attempt = 0; attempt < 80; ++attempt) {
        kv.clear();
        int mmax[3];
        for (int d = 0; d < 3; ++d) mmax[d] = (int)std::floor(kc * h->L[d] / (2.0 * kPi));
        for (int mx = 0; mx <= mmax[0]; ++mx)
            for (int my = -mmax[1]; my <= mmax[1]; ++my)
                for (int mz = -mmax[2]; mz <= mmax[2]; ++mz) {
                    if (mx == 0 && (my < 0 || (my == 0 && mz <= 0))) continue;
                    const double kx = 2 * kPi * mx / h->L[0], ky = 2 * kPi * my / h->L[1], kz = 2 * kPi * mz / h->L[2];
                    const double k2 = kx * kx + ky * ky + kz * kz, k = std::sqrt(k2);
                    if (k >= kc) continue;
                    const double j0 = std::sin(k) / k;
                    const double w = 2.0 * j0 * j0 * std::exp(-k2 / (4.0 * xi * xi)) / (k2 * V);
                    kv.push_back(make_float4((float)mx, (float)my, (float)mz, (float)std::sqrt(w)));
                }
        if ((int)kv.size() <= max_modes) break;
        kc *= 0.95;
    }
    const int nmodes = (int)kv.size();
    std::vector<int4> rows;  // runs of consecutive m_z at fixed (m_x, m_y): (mx, my, mz0, first mode)
    for (int m = 0; m < nmodes; ++m) {
        const int mx = (int)kv[m].x, my = (int)kv[m].y, mz = (int)kv[m].z;
        if (m == 0 || mx != (int)kv[m - 1].x || my != (int)kv[m - 1].y || mz != (int)kv[m - 1].z + 1)
            rows.push_back(make_int4(mx, my, mz, m));
    }
    const int nrows = (int)rows.size();
    const int K2 = std::max(16, (2 * nmodes + 15) / 16 * 16);
    // dense: padded order (identity on the padding)
    const int np = sparse ? nc : (nc + GT - 1) / GT * GT;
    const int K = cs.pcg_iters;
    const int nspmv = (nbc + kSpmvWarpsC - 1) / kSpmvWarpsC, nvec = (nbc + kVecThreads - 1) / kVecThreads;
    CR_TRY(grow(h, &cs.kv, cs.cap_kv, (size_t)std::max(nmodes, 1), moved));
    CR_TRY(grow(h, &cs.rows, cs.cap_rows, (size_t)std::max(nrows, 1), moved));
    CR_TRY(grow(h, &cs.F, cs.cap_F, (size_t)nc * K2, moved));
    const int nchunk = (nc + kColRows - 1) / kColRows;
    CR_TRY(grow(h, &cs.fpart, cs.cap_fpart, (size_t)nchunk * K2, moved));
    if (!sparse) {
        CR_TRY(grow(h, &cs.C, cs.cap_C, (size_t)np * np, moved));
        CR_TRY(grow(h, &cs.Ci, cs.cap_Ci, (size_t)np * np, moved));
        CR_TRY(grow(h, &cs.R, cs.cap_R, (size_t)NB * np, moved));
        CR_TRY(grow(h, &cs.Fc, cs.cap_Fc, (size_t)np * NB, moved));
        CR_TRY(grow(h, &cs.Dinv, cs.cap_Dinv, (size_t)NB * NB, moved));
    } else {
        CR_TRY(grow(h, &cs.Cblk, cs.cap_Cblk, (size_t)npairs * 9, moved));
        CR_TRY(grow(h, &cs.Dblk, cs.cap_Dblk, (size_t)nbc * 9, moved));
        CR_TRY(grow(h, &cs.pr, cs.cap_pr, (size_t)np, moved));
        CR_TRY(grow(h, &cs.pz, cs.cap_pz, (size_t)np, moved));
        CR_TRY(grow(h, &cs.pp, cs.cap_pp, (size_t)np, moved));
        CR_TRY(grow(h, &cs.pq, cs.cap_pq, (size_t)np, moved));
        CR_TRY(grow(h, &cs.pu, cs.cap_pu, (size_t)K2, moved));
        CR_TRY(grow(h, &cs.part_pq, cs.cap_part_pq, (size_t)K * nspmv, moved));
        CR_TRY(grow(h, &cs.part_rz, cs.cap_part_rz, (size_t)(K + 1) * nvec, moved));
    }
    CR_TRY(grow(h, &cs.g, cs.cap_g, (size_t)np, moved));  // zero beyond nc: the padded GEMV rows
    CR_TRY(grow(h, &cs.y, cs.cap_y, (size_t)np, moved));
    CR_TRY(grow(h, &cs.u, cs.cap_u, (size_t)K2, moved));
    CR_TRY(grow(h, &cs.t, cs.cap_t, n1, moved));
    if (nmodes > 0) {
        CR_CUDA(h, cudaMemcpyAsync(cs.kv, kv.data(), nmodes * sizeof(float4), cudaMemcpyHostToDevice, h->stream));
        CR_CUDA(h, cudaMemcpyAsync(cs.rows, rows.data(), nrows * sizeof(int4), cudaMemcpyHostToDevice, h->stream));
    }
    // threads per body CTA: the largest body rounded up to whole warps
    int max_n = 0;
    for (int b = 0; b < B; ++b) max_n = std::max(max_n, h->h_body_start[b + 1] - h->h_body_start[b]);
    const int bs = std::min(256, std::max(32, (max_n + 31) / 32 * 32));
    // two threads per bead when one pass covers every body (more warps for the latency-
    // bound rotation chains of the wave rows)
    const int model_split = max_n <= bs ? 2 : 1;
    int max_pairs = 0;
    for (int a = 0; a < nbc; ++a) max_pairs = std::max(max_pairs, pcount[a]);
    const size_t model_smem =
        ((size_t)nrows + (nmodes + 1) / 2) * sizeof(float4) + (size_t)max_pairs * 2 * sizeof(double2) +
        (size_t)(model_split - 1) * bs * sizeof(double);
    if (model_smem > 48 * 1024)
        CR_CUDA(h, cudaFuncSetAttribute(coarse_model_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)model_smem));
    CR_CUDA(h, cudaMemsetAsync(cs.F, 0, (size_t)nc * K2 * sizeof(float), h->stream));
    CR_CUDA(h, cudaMemsetAsync(cs.g, 0, (size_t)np * sizeof(double), h->stream));
    CR_CUDA(h, cudaMemsetAsync(cs.y, 0, (size_t)np * sizeof(double), h->stream));
    if (nmodes > 0) {
        coarse_wave_basis_kernel<<<nbc, 128, 0, h->stream>>>(nmodes, cs.kv, cs.cbody, h->d_body_start,
                                                             h->d_body_members, h->m64.pos, Linv, cs.zq, K2,
                                                             cs.F);
        CR_LAUNCH(h, "coarse_wave_basis_kernel");
    }
    // dense: C = F F^T + real-space blocks (+ self), padded with the identity;
    // sparse: the near-pair blocks only
    if (!sparse) {
        dim3 tg((nc + 63) / 64, (nc + 63) / 64);
        syrk_kernel<<<tg, 256, 0, h->stream>>>(nc, K2, cs.F, K2, cs.C, np);
        CR_LAUNCH(h, "syrk_kernel");
    }
    double *cblk = sparse ? cs.Cblk : nullptr;
    RealArgs ra;
    double max_rad = 0.0;
    for (int b : cbody) max_rad = std::max(max_rad, cent[b].w);
    bool shift = true;
    for (int d = 0; d < 3; ++d) {
        ra.Ld[d] = h->L[d];
        ra.L[d] = (float)h->L[d];
        ra.Linv[d] = (float)(1.0 / h->L[d]);
        shift = shift && h->L[d] >= 2.0 * (h->d.rcut + 2.0 * max_rad) + 1e-6;
    }
    ra.rc = (float)h->d.rcut;
    ra.rc2 = (float)(h->d.rcut * h->d.rcut);
    ra.rmin2 = (float)(h->d.dr * h->d.dr);
    ra.dr = (float)h->d.dr;
    ra.inv_dr = (float)(1.0 / h->d.dr);
    ra.scale = (float)(h->d.n_table / (h->d.rcut - h->d.dr));
    ra.ntab = h->d.n_table;
    ra.selfc = h->d.selfcoeff;
    if (shift)
        coarse_real_kernel<true><<<(unsigned)npairs, bs, 0, h->stream>>>(
            cs.pair_a, cs.pair_b, cs.woff, cs.cbody, h->d_body_start, h->d_body_members, h->m64.pos, cs.cent, cs.zq,
            h->m32.phiq, ra, np, cs.W, cs.C, cblk);
    else
        coarse_real_kernel<false><<<(unsigned)npairs, bs, 0, h->stream>>>(
            cs.pair_a, cs.pair_b, cs.woff, cs.cbody, h->d_body_start, h->d_body_members, h->m64.pos, cs.cent, cs.zq,
            h->m32.phiq, ra, np, cs.W, cs.C, cblk);
    CR_LAUNCH(h, "coarse_real_kernel");
    CR_CUDA(h, cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    if (!sparse) {
        symmetrise_kernel<<<blocks_for((long)nc * nc, 256), 256, 0, h->stream>>>(nc, cs.C, np);
        CR_LAUNCH(h, "symmetrise_kernel");
        pad_identity_kernel<<<blocks_for((long)np * np, 256), 256, 0, h->stream>>>(nc, np, cs.C);
        CR_LAUNCH(h, "pad_identity_kernel");

        // C^-1: FP32 copy inverted in place
        to_float_kernel<<<blocks_for((long)np * np, 256), 256, 0, h->stream>>>((long long)np * np, cs.C, cs.Ci);
        CR_LAUNCH(h, "to_float_kernel");
        for (int k0 = 0; k0 < np; k0 += NB) {
            gj_pivot_kernel<<<1, kPivThreads, 0, h->stream>>>(k0, np, cs.Ci, cs.Dinv, h->d_flag);
            CR_LAUNCH(h, "gj_pivot_kernel");
            gj_panel_kernel<<<np / NB, 256, 0, h->stream>>>(k0, np, cs.Ci, cs.Dinv, cs.R, cs.Fc);
            CR_LAUNCH(h, "gj_panel_kernel");
            const int nt = np / GT;
            gj_update_kernel<<<nt * (nt + 1) / 2, 256, 0, h->stream>>>(k0, np, cs.Ci, cs.R, cs.Fc);
            CR_LAUNCH(h, "gj_update_kernel");
        }
        mirror_upper_kernel<<<blocks_for((long)np * np, 256), 256, 0, h->stream>>>(np, cs.Ci);
        CR_LAUNCH(h, "mirror_upper_kernel");
    } else {
        block_jacobi_kernel<<<blocks_for(nbc, 128), 128, 0, h->stream>>>(nbc, cs.phead, cs.pcount, cs.pair_b, cs.Cblk,
                                                                          cs.F, K2, cs.Dblk, h->d_flag);
        CR_LAUNCH(h, "block_jacobi_kernel");
    }
    int bad = 0;
    CR_CUDA(h, cudaMemcpyAsync(&bad, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    if (moved) {  // captured solver steps hold the old addresses
        h->kry.exec_gen[0] = h->kry.exec_gen[1] = -1;
    }
    cs.gen = h->geo_gen;
    cs.nbc = nbc;
    cs.nc = nc;
    cs.np = np;
    cs.nmodes = nmodes;
    cs.nrows = nrows;
    cs.sparse = sparse;
    cs.nspmv = nspmv;
    cs.nvec = nvec;
    cs.bs = bs;
    cs.model_smem = model_smem;
    cs.model_split = model_split;
    cs.K2 = K2;
    cs.npairs = npairs;
    cs.kc = kc;
    cs.failed = bad != 0;
    cs.active = !cs.failed;
    return CR_OK;
}

// The two-level preconditioner of a lockstep batch: the stages of coarse_apply, each one
// launch over the replicas (a replica without an active coarse level only takes the
// conductor response of its input).  Replicas share the model kernel's launch shape
// (the largest body rounded to whole warps, two threads per bead), so the batch requires
// it to be the same for all of them.
int batch_coarse_attrs(cr_batch *bt) {
    static size_t set = 0;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (bt->model_smem > 48 * 1024 && bt->model_smem > set) {
        CR_TRY(batch_check(bt, cudaFuncSetAttribute(model_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    (int)bt->model_smem),
                           "model_batch_kernel attribute"));
        set = bt->model_smem;
    }
    return CR_OK;
}

int batch_coarse(cr_batch *bt, const int *mask, int xin, int zout, cudaStream_t s) {
    const int split = bt->model_threads > 0 ? bt->model_split : 1;
    if (bt->n_items[BL_CBODIES] > 0) {
        restrict_batch_kernel<<<bt->n_items[BL_CBODIES], 128, 0, s>>>(bt->d_reps, bt->d_items[BL_CBODIES], mask, xin);
        ++bt->launches;
        CR_TRY(batch_check(bt, cudaGetLastError(), "restrict_batch_kernel"));
    }
    if (bt->n_items[BL_GEMV] > 0) {
        gemv_batch_kernel<<<bt->n_items[BL_GEMV], 256, 0, s>>>(bt->d_reps, bt->d_items[BL_GEMV], mask);
        ++bt->launches;
        CR_TRY(batch_check(bt, cudaGetLastError(), "gemv_batch_kernel"));
    }
    if (bt->n_items[BL_FCHUNK] > 0) {
        fpart_batch_kernel<<<bt->n_items[BL_FCHUNK], 256, 0, s>>>(bt->d_reps, bt->d_items[BL_FCHUNK], mask);
        ++bt->launches;
        CR_TRY(batch_check(bt, cudaGetLastError(), "fpart_batch_kernel"));
        freduce_batch_kernel<<<bt->n_items[BL_FCOL], 256, 0, s>>>(bt->d_reps, bt->d_items[BL_FCOL], mask);
        ++bt->launches;
        CR_TRY(batch_check(bt, cudaGetLastError(), "freduce_batch_kernel"));
    }
    if (bt->n_items[BL_BODIES] > 0 && bt->n_items[BL_CBODIES] > 0) {
        model_batch_kernel<<<bt->n_items[BL_BODIES], bt->model_threads, bt->model_smem, s>>>(
            bt->d_reps, bt->d_items[BL_BODIES], mask, xin, split);
        ++bt->launches;
        CR_TRY(batch_check(bt, cudaGetLastError(), "model_batch_kernel"));
    }
    CR_TRY(batch_conductor(bt, mask, xin, true, zout, s));
    if (bt->n_items[BL_CBODIES] > 0) {
        prolong_batch_kernel<<<bt->n_items[BL_CBODIES], 128, 0, s>>>(bt->d_reps, bt->d_items[BL_CBODIES], mask, zout);
        ++bt->launches;
        CR_TRY(batch_check(bt, cudaGetLastError(), "prolong_batch_kernel"));
    }
    return CR_OK;
}

int coarse_apply(cr_handle *h, const double *x, double *z) {
    const CoarseSpace &cs = h->coarse;
    if (!cs.active) return conductor_apply(h, x, z);
    const int N = h->N, B = h->B;
    const double3 Linv = make_double3(1.0 / h->L[0], 1.0 / h->L[1], 1.0 / h->L[2]);
    coarse_restrict_kernel<<<cs.nbc, 128, 0, h->stream>>>(N, cs.cbody, h->d_body_start, h->d_body_members, cs.zq,
                                                           cs.zp, x, cs.g);
    CR_LAUNCH(h, "coarse_restrict_kernel");
    if (!cs.sparse) {
        coarse_gemv_kernel<<<blocks_for((long)cs.nc * 32, 256), 256, 0, h->stream>>>(cs.nc, cs.np, cs.Ci, cs.g,
                                                                                     cs.y);
        CR_LAUNCH(h, "coarse_gemv_kernel");
    } else {  // y ~= -C^-1 g by pcg_iters block-Jacobi CG steps
        const int K = cs.pcg_iters, nv = cs.nvec, ns = cs.nspmv;
        pcg_init_kernel<<<nv, kVecThreads, 0, h->stream>>>(cs.nbc, cs.Dblk, cs.g, cs.y, cs.pr, cs.pz, cs.pp,
                                                            cs.part_rz);
        CR_LAUNCH(h, "pcg_init_kernel");
        for (int it = 0; it < K; ++it) {
            if (cs.nmodes > 0) {
                const int nchunk = (cs.nc + kColRows - 1) / kColRows;
                fcol_partial_kernel<<<nchunk, 256, 0, h->stream>>>(cs.nc, cs.K2, cs.F, cs.pp, cs.fpart);
                CR_LAUNCH(h, "fcol_partial_kernel");
                fcol_reduce_kernel<double><<<blocks_for(32L * cs.K2, 256), 256, 0, h->stream>>>(
                    nchunk, cs.K2, cs.fpart, 0, nullptr, cs.pu);
                CR_LAUNCH(h, "fcol_reduce_kernel");
            }
            pcg_spmv_kernel<<<ns, kSpmvWarpsC * 32, 0, h->stream>>>(cs.nbc, cs.phead, cs.pcount, cs.pair_b, cs.Cblk,
                                                                     cs.F, cs.nmodes > 0 ? cs.K2 : 0, cs.pu, cs.pp,
                                                                     cs.pq, cs.part_pq + (size_t)it * ns);
            CR_LAUNCH(h, "pcg_spmv_kernel");
            pcg_update_kernel<<<nv, kVecThreads, 0, h->stream>>>(cs.nbc, ns, cs.part_pq + (size_t)it * ns, nv,
                                                                  cs.part_rz + (size_t)it * nv, cs.Dblk, cs.pp, cs.pq,
                                                                  cs.y, cs.pr, cs.pz, cs.part_rz + (size_t)(it + 1) * nv);
            CR_LAUNCH(h, "pcg_update_kernel");
            if (it + 1 < K) {
                pcg_dir_kernel<<<blocks_for(3L * cs.nbc, kVecThreads), kVecThreads, 0, h->stream>>>(
                    cs.nbc, nv, cs.part_rz + (size_t)it * nv, cs.part_rz + (size_t)(it + 1) * nv, cs.pz, cs.pp);
                CR_LAUNCH(h, "pcg_dir_kernel");
            }
        }
    }
    if (cs.nmodes > 0) {
        const int nchunk = (cs.nc + kColRows - 1) / kColRows;
        fcol_partial_kernel<<<nchunk, 256, 0, h->stream>>>(cs.nc, cs.K2, cs.F, cs.y, cs.fpart);
        CR_LAUNCH(h, "fcol_partial_kernel");
        fcol_reduce_kernel<float><<<blocks_for(32L * cs.K2, 256), 256, 0, h->stream>>>(nchunk, cs.K2, cs.fpart, cs.nmodes,
                                                                               cs.kv, cs.u);
        CR_LAUNCH(h, "fcol_reduce_kernel");
    }
    coarse_model_kernel<<<B, cs.bs * cs.model_split, cs.model_smem, h->stream>>>(N, cs.nmodes, cs.nrows, cs.rows, cs.cidx,
                                                                 h->d_body_start, h->d_body_members, h->m64.pos,
                                                                 Linv, cs.zq, cs.zp, cs.phead, cs.pcount, cs.pair_b,
                                                                 cs.woff, cs.W, cs.u, h->d.selfcoeff, cs.y, x, cs.t,
                                                                 cs.model_split);
    CR_LAUNCH(h, "coarse_model_kernel");
    CR_TRY(conductor_apply(h, cs.t, z));
    coarse_prolong_kernel<<<cs.nbc, 128, 0, h->stream>>>(N, cs.cbody, h->d_body_start, h->d_body_members, cs.zq,
                                                          cs.zp, cs.y, z);
    CR_LAUNCH(h, "coarse_prolong_kernel");
    return CR_OK;
}

}  // namespace cr
