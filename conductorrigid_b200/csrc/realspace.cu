// realspace.cu -- real-space part of the operator and of the force pass
// (ConductorRigid.cu:469-664).
//
// The reference walks a per-bead neighbour list in every matrix-vector product and
// re-evaluates the tabulated kernel for each pair.  Here the geometry is fixed for a
// whole solve, so the real-space operator is built once per solve as a symmetric
// block-sparse matrix and every GMRES iteration streams it:
//
//  * clusters: beads sorted along a Morton curve of the box, cut into clusters of 32
//    (the last one padded);
//  * cluster pairs (I, J), both orders, whose bounding boxes come within rc under any
//    periodic image, found once per solve;
//  * per pair a 32x32 bit mask (row i, bit j) of the bead pairs with
//    dr^2 <= d^2 < rc^2 under the minimum image (ConductorRigid.cu:536-540), and the
//    values T(d_ij) of just those pairs with the table index
//    floor(Ntable (d - dr)/(rc - dr)) and linear weight d/dr - index - 1 of
//    ConductorRigid.cu:549-554, evaluated in FP64 and stored in the operator
//    precision (the 32x32 blocks of a 4-unit cutoff are only 20-35% full, so the mask
//    keeps the streamed bytes near one value per interacting pair).  The values of a
//    pair are stored lane-interleaved: the k-th value of row i at k*32 + i, rows padded
//    with zeros to the pair's longest row, so that every load is one coalesced warp
//    load;
//  * the product y_I = sum_J B_IJ x_J, the pairs of cluster I split over the warps of
//    one CTA: lane i takes the k-th set bit j of its row, multiplies the k-th value by
//    x_J[j] fetched with a warp shuffle; the partial sums are added in warp order, so
//    there are no atomics and the sum order is fixed.
//
// The force pass (once per solve) evaluates the gradient table on the fly over the same
// cluster pairs in FP64.
#include <cub/cub.cuh>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "cr_internal.cuh"

namespace cr {

namespace {

constexpr int CS = 32;  // beads per cluster

struct RSBuild {
    double L[3], Linv[3];
    double rc, rc2, rmin2, dr, inv_dr, scale;  // scale = ntab / (rc - dr)
    int ntab;
};

__device__ __forceinline__ double mimg(double dx, double L, double Linv) { return dx - L * rint(dx * Linv); }

// Morton key of a position on a 1024^3 lattice of the box.
__device__ __forceinline__ unsigned spread_bits(unsigned v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void morton_kernel(int N, const double4 *__restrict__ pos, double Lx, double Ly, double Lz, int *key,
                              int *iota) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double4 p = pos[i];
    const int ix = min(max((int)((p.x / Lx + 0.5) * 1024.0), 0), 1023);
    const int iy = min(max((int)((p.y / Ly + 0.5) * 1024.0), 0), 1023);
    const int iz = min(max((int)((p.z / Lz + 0.5) * 1024.0), 0), 1023);
    key[i] = (int)((spread_bits(ix) << 2) | (spread_bits(iy) << 1) | spread_bits(iz));
    iota[i] = i;
}

// Cluster members (padded with -1), centre and half extent (relative to the first
// member under the minimum image, so clusters that cross the boundary stay compact).
__global__ void cluster_kernel(int N, int nclus, const int *__restrict__ sorted, const double4 *__restrict__ pos,
                               RSBuild c, int *members, double4 *centre, double4 *extent) {
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (I >= nclus) return;
    const int k = I * CS + lane;
    const int i = k < N ? sorted[k] : -1;
    members[k] = i;
    const int i0 = sorted[I * CS];
    const double4 p0 = pos[i0];
    double r[3] = {0, 0, 0};
    if (i >= 0) {
        const double4 p = pos[i];
        r[0] = mimg(p.x - p0.x, c.L[0], c.Linv[0]);
        r[1] = mimg(p.y - p0.y, c.L[1], c.Linv[1]);
        r[2] = mimg(p.z - p0.z, c.L[2], c.Linv[2]);
    }
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = i >= 0 ? r[d] : 1e300;
        hi[d] = i >= 0 ? r[d] : -1e300;
        for (int o = 16; o > 0; o >>= 1) {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
    }
    if (lane == 0) {
        centre[I] = make_double4(p0.x + 0.5 * (lo[0] + hi[0]), p0.y + 0.5 * (lo[1] + hi[1]),
                                 p0.z + 0.5 * (lo[2] + hi[2]), 0.0);
        extent[I] = make_double4(0.5 * (hi[0] - lo[0]), 0.5 * (hi[1] - lo[1]), 0.5 * (hi[2] - lo[2]), 0.0);
    }
}

// Smallest bounding-box gap between clusters I and J over the periodic images.
__device__ __forceinline__ double box_gap2(const double4 &ci, const double4 &ei, const double4 &cj, const double4 &ej,
                                           const RSBuild &c) {
    const double dc[3] = {cj.x - ci.x, cj.y - ci.y, cj.z - ci.z};
    const double es[3] = {ei.x + ej.x, ei.y + ej.y, ei.z + ej.z};
    double g2 = 0.0;
    for (int d = 0; d < 3; ++d) {
        const double m = mimg(dc[d], c.L[d], c.Linv[d]);
        double best = 1e300;
        for (int s = -1; s <= 1; ++s) {
            const double v = fabs(m + s * c.L[d]) - es[d];
            best = fmin(best, v > 0.0 ? v : 0.0);
        }
        g2 += best * best;
    }
    return g2;
}

// One warp per cluster I scans every J; FILL writes J in ascending order.
template <bool FILL>
__global__ void pair_search_kernel(int nclus, const double4 *__restrict__ centre, const double4 *__restrict__ extent,
                                   RSBuild c, int *count, const long long *__restrict__ head, int *pair_j) {
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (I >= nclus) return;
    const double4 ci = centre[I], ei = extent[I];
    int n = 0;
    const long long h0 = FILL ? head[I] : 0;
    for (int base = 0; base < nclus; base += 32) {
        const int J = base + lane;
        bool hit = false;
        // a bead pair at exactly the cutoff can make two clusters' box gap equal rc: the
        // test is widened by a relative 1e-9 so that rounding never drops such a cluster
        // pair (the masks then decide every bead pair exactly)
        if (J < nclus) hit = J == I || box_gap2(ci, ei, centre[J], extent[J], c) < c.rc2 * (1.0 + 1e-9);
        const unsigned mask = __ballot_sync(0xffffffffu, hit);
        if (FILL && hit) pair_j[h0 + n + __popc(mask & ((1u << lane) - 1u))] = J;
        n += __popc(mask);
    }
    if (!FILL && lane == 0) count[I] = n;
}

__global__ void pair_owner_kernel(int nclus, const long long *__restrict__ head, const int *__restrict__ count,
                                  int *pair_i) {
    const int I = blockIdx.x;
    if (I >= nclus) return;
    for (int k = threadIdx.x; k < count[I]; k += blockDim.x) pair_i[head[I] + k] = I;
}

__device__ __forceinline__ double table_lerp64(const double2 *__restrict__ tab, const RSBuild &c, double d) {
    int ind = (int)floor((d - c.dr) * c.scale);
    ind = min(max(ind, 0), c.ntab - 1);
    const double lin = d * c.inv_dr - ind - 1.0;
    const double2 e = tab[ind];
    return e.x + (e.y - e.x) * lin;
}

// 1/sqrt(d2) for d2 > 0 in FP64: the FP32 estimate refined by two Newton-Raphson steps
// for the reciprocal square root, y <- y (3 - d2 y^2) / 2 (relative error squared per
// step: ~1e-7 -> ~1e-14 -> the FP64 rounding level).
__device__ __forceinline__ double rsqrt64(double d2) {
    double y = (double)rsqrtf((float)d2);
    y = y * (1.5 - 0.5 * d2 * y * y);
    y = y * (1.5 - 0.5 * d2 * y * y);
    return y;
}

// Squared minimum-image distance with every operation rounded separately (no fused
// multiply-add), the arithmetic of the oracle's neighbour test: pairs at exactly the
// cutoff -- antipodal beads of a sphere of radius rc/2 -- are decided the same way.
__device__ __forceinline__ double dist2_exact(const double4 &a, const double4 &b, const RSBuild &c) {
    double e[3] = {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)};
    for (int d = 0; d < 3; ++d) e[d] = __dsub_rn(e[d], __dmul_rn(c.L[d], rint(__dmul_rn(e[d], c.Linv[d]))));
    return __dadd_rn(__dadd_rn(__dmul_rn(e[0], e[0]), __dmul_rn(e[1], e[1])), __dmul_rn(e[2], e[2]));
}

// Bit masks of the in-range bead pairs of every cluster pair (row i = bead i of I,
// bit j = bead j of J) and the stored slots of the pair (32 x its longest row).
// The test runs on the FP32 copies of the positions; only a pair whose FP32 squared
// distance lies within `band` of rc^2 (or below 2 dr^2 + band) is decided again in FP64,
// exactly as the oracle decides it.  `band` is ten times a bound on the FP32 error of
// d^2 for |d| <= rc in a box of edge L (positions rounded to FP32: |error of dx| <= 2e-7 L),
// so the masks equal the FP64 ones bit for bit.
__global__ void pair_mask_kernel(long long npairs, const int *__restrict__ pair_i, const int *__restrict__ pair_j,
                                 const int *__restrict__ members, const double4 *__restrict__ pos,
                                 const float4 *__restrict__ pos32, RSBuild c, float3 L32, float3 Linv32, float rc2,
                                 float band, float low, unsigned *__restrict__ masks, int *__restrict__ nnz,
                                 unsigned long long *__restrict__ bits, const double4 *__restrict__ centre,
                                 const double4 *__restrict__ extent, float4 *__restrict__ pshift) {
    const long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= npairs) return;
    const int I = pair_i[p], J = pair_j[p];
    const int bi = members[I * CS + lane];
    const int bj = members[J * CS + lane];
    const float4 pi = bi >= 0 ? pos32[bi] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 pjl = bj >= 0 ? pos32[bj] : make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned m = 0;
    for (int j = 0; j < CS; ++j) {
        const int vj = __shfl_sync(0xffffffffu, bj, j);
        const float xj = __shfl_sync(0xffffffffu, pjl.x, j);
        const float yj = __shfl_sync(0xffffffffu, pjl.y, j);
        const float zj = __shfl_sync(0xffffffffu, pjl.z, j);
        if (bi >= 0 && vj >= 0) {
            float dx = pi.x - xj, dy = pi.y - yj, dz = pi.z - zj;
            dx -= L32.x * rintf(dx * Linv32.x);
            dy -= L32.y * rintf(dy * Linv32.y);
            dz -= L32.z * rintf(dz * Linv32.z);
            const float d2 = dx * dx + dy * dy + dz * dz;
            bool in;
            if (d2 > rc2 + band) {
                in = false;
            } else if (d2 < rc2 - band && d2 > low) {
                in = true;
            } else {  // near a boundary: the FP64 decision, rounded as the oracle rounds it
                const double4 a = pos[bi], b = pos[vj];
                const double e2 = dist2_exact(a, b, c);
                in = e2 < c.rc2 && e2 >= c.rmin2;
            }
            if (in) m |= 1u << j;
        }
    }
    masks[p * CS + lane] = m;
    int n = __popc(m), tot = n;
    for (int o = 16; o > 0; o >>= 1) {
        n = max(n, __shfl_xor_sync(0xffffffffu, n, o));
        tot += __shfl_xor_sync(0xffffffffu, tot, o);
    }
    if (lane == 0) {
        nnz[p] = n * CS;  // stored slots: longest row times 32 lanes
        atomicAdd(bits, (unsigned long long)tot);
        // offset of the cluster centres under the minimum image, and whether the bead
        // offsets then need no further image: rc + 2 (e_I + e_J) < L/2 along every axis
        const double4 cI = centre[I], cJ = centre[J], eI = extent[I], eJ = extent[J];
        const bool direct = c.rc + 2.0 * (eI.x + eJ.x) < 0.5 * c.L[0] - 1e-3 &&
                            c.rc + 2.0 * (eI.y + eJ.y) < 0.5 * c.L[1] - 1e-3 &&
                            c.rc + 2.0 * (eI.z + eJ.z) < 0.5 * c.L[2] - 1e-3;
        pshift[p] = make_float4((float)mimg(cJ.x - cI.x, c.L[0], c.Linv[0]), (float)mimg(cJ.y - cI.y, c.L[1], c.Linv[1]),
                                (float)mimg(cJ.z - cI.z, c.L[2], c.Linv[2]), direct ? 1.f : 0.f);
    }
}

__device__ __forceinline__ int warp_exclusive_scan(int v, int lane) {
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    return incl - v;
}

// Values T(d_ij) of the set mask bits in the operator precision, lane-interleaved:
// the k-th set bit of row i at voff + k*32 + i, zeros after the row's last bit.
// With R2 = double (and R = float) one pass writes both precisions' values.
template <typename R, typename R2 = void>
__global__ void pair_values_kernel(long long npairs, const int *__restrict__ pair_i, const int *__restrict__ pair_j,
                                   const int *__restrict__ members, const double4 *__restrict__ pos,
                                   const double2 *__restrict__ tab, RSBuild c, const unsigned *__restrict__ masks,
                                   const long long *__restrict__ voff, const int *__restrict__ slots,
                                   R *__restrict__ vals, double *__restrict__ vals2 = nullptr) {
    constexpr bool BOTH = std::is_same<R2, double>::value;
    const long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= npairs) return;
    const int I = pair_i[p], J = pair_j[p];
    const int bi = members[I * CS + lane];
    const int bj = members[J * CS + lane];
    const double4 pi = bi >= 0 ? pos[bi] : make_double4(0, 0, 0, 0);
    const double4 pjl = bj >= 0 ? pos[bj] : make_double4(0, 0, 0, 0);
    const unsigned m = masks[p * CS + lane];
    R *out = vals + voff[p] + lane;
    double *out2 = BOTH ? vals2 + voff[p] + lane : nullptr;
    // lane i walks its own set bits (the k-th bit j at step k), fetching bead j's position
    // from lane j; lanes past their last bit write the zero padding of the slot
    const int rows = slots[p] / CS;
    unsigned mm = m;
    for (int k = 0; k < rows; ++k) {
        const bool has = mm != 0;
        const int j = has ? __ffs(mm) - 1 : 0;
        mm &= mm - 1;
        const double xj = __shfl_sync(0xffffffffu, pjl.x, j);
        const double yj = __shfl_sync(0xffffffffu, pjl.y, j);
        const double zj = __shfl_sync(0xffffffffu, pjl.z, j);
        double t = 0.0;
        if (has) {
            const double dx = mimg(pi.x - xj, c.L[0], c.Linv[0]);
            const double dy = mimg(pi.y - yj, c.L[1], c.Linv[1]);
            const double dz = mimg(pi.z - zj, c.L[2], c.Linv[2]);
            const double d2 = dx * dx + dy * dy + dz * dz;
            t = table_lerp64(tab, c, d2 * rsqrt64(d2));
        }
        out[(size_t)k * CS] = (R)t;
        if (BOTH) out2[(size_t)k * CS] = t;
    }
}

// Charges in cluster order (0 for padding), so that a warp reads a cluster's charges
// with one coalesced load.
template <typename R>
__global__ void gather_cluster_kernel(int n, const int *__restrict__ members, const R *__restrict__ q,
                                      R *__restrict__ qc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = members[k];
    qc[k] = i >= 0 ? q[i] : (R)0;
}

// y_I = sum_J B_IJ x_J for cluster I (one CTA of W warps), combined with the wave-space
// part and the self term: out_i = Phi_body(i) - (phik_i + self q_i + y_i), or the bare
// sum when phi_body is NULL.  Warp w takes pairs w, w+W, ...; lane i consumes the set
// bits of its mask row in order, the k-th against the coalesced load of slot k, with
// x_J[j] from a shuffle.  Up to U slots are loaded before they are used; the next
// pair's metadata is fetched while the current one is summed.  The W partial sums are
// added in warp order, so the result does not depend on scheduling.
// FP32: six CTAs per SM (at most 40 registers; 48 warps of loads in flight, 0.864 ->
// 0.835 ms per application at 162k charges; 32 registers spill and lose it again).
template <typename R, int W, int U>
__global__ void __launch_bounds__(W * 32, sizeof(R) == 4 ? 6 : 1) pair_spmv_kernel(int nclus, const long long *__restrict__ head,
                                                           const int *__restrict__ count,
                                                           const int *__restrict__ pair_j,
                                                           const int *__restrict__ members,
                                                           const unsigned *__restrict__ masks,
                                                           const long long *__restrict__ voff,
                                                           const int *__restrict__ slots,
                                                           const R *__restrict__ vals, const R *__restrict__ qc,
                                                           const R *__restrict__ q, const R *__restrict__ phik,
                                                           double selfc, const double *__restrict__ phi_body,
                                                           const uint32_t *__restrict__ body,
                                                           double *__restrict__ out) {
    __shared__ R part[W][CS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int I = blockIdx.x;
    R yI = 0;
    const long long h0 = head[I];
    const int n = count[I];
    int J = 0, rows = 0;
    unsigned m0 = 0;
    long long off = 0;
    R xJ = 0;
    if (w < n) {
        J = pair_j[h0 + w];
        m0 = masks[(h0 + w) * CS + lane];
        off = voff[h0 + w];
        rows = slots[h0 + w] / CS;
        xJ = qc[J * CS + lane];
    }
    for (int k = w; k < n; k += W) {
        const R *v = vals + off + lane;
        unsigned m = m0;
        const R xcur = xJ;
        const int rcur = rows;
        if (k + W < n) {
            const long long p1 = h0 + k + W;
            J = pair_j[p1];
            m0 = masks[p1 * CS + lane];
            off = voff[p1];
            rows = slots[p1] / CS;
            xJ = qc[J * CS + lane];
        }
        const int own = __popc(m);  // slots past the end of this lane's row hold zeros: skip them
        for (int base = 0; base < rcur; base += U) {
            R t[U];
#pragma unroll
            for (int u = 0; u < U; ++u) t[u] = base + u < own ? __ldg(v + (size_t)(base + u) * CS) : (R)0;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = m ? __ffs(m) - 1 : 0;
                m &= m - 1;
                yI += t[u] * __shfl_sync(0xffffffffu, xcur, j);
            }
        }
    }
    part[w][lane] = yI;
    __syncthreads();
    if (w == 0) {
        R tot = 0;
#pragma unroll
        for (int v = 0; v < W; ++v) tot += part[v][lane];
        const int bi = members[I * CS + lane];
        if (bi >= 0) {
            const double total = (double)phik[bi] + selfc * (double)q[bi] + (double)tot;
            out[bi] = phi_body ? phi_body[body[bi]] - total : total;
        }
    }
}

constexpr int kSpmvWarps = 8;

// Bead offsets from their cluster's centre in FP32 (minimum image; 0 for padding).
__global__ void cluster_offsets_kernel(int n, const int *__restrict__ members, const double4 *__restrict__ pos,
                                       const double4 *__restrict__ centre, RSBuild c, float4 *__restrict__ off) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = members[k];
    float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
    if (i >= 0) {
        const double4 p = pos[i], cc = centre[k / CS];
        o.x = (float)mimg(p.x - cc.x, c.L[0], c.Linv[0]);
        o.y = (float)mimg(p.y - cc.y, c.L[1], c.Linv[1]);
        o.z = (float)mimg(p.z - cc.z, c.L[2], c.Linv[2]);
    }
    off[k] = o;
}

// Tabulated kernel in FP32 from the shared-memory table: index floor((d - dr) Ntable /
// (rc - dr)) clamped into the table, weight d/dr - index - 1 (ConductorRigid.cu:549-554).
__device__ __forceinline__ float table_lerp32(const float2 *__restrict__ tab, float d2, int ntab, float scale,
                                              float dr, float inv_dr) {
    const float d = d2 * rsqrtf(d2);
    int ind = (int)((d - dr) * scale);  // truncation = floor for d >= dr; FP32 rounding below dr gives 0
    ind = min(max(ind, 0), ntab - 1);
    const float lin = fmaf(d, inv_dr, -(float)(ind + 1));
    const float2 e = tab[ind];
    return fmaf(e.y - e.x, lin, e.x);
}

// The FP32 product y_I = sum_J B_IJ x_J with the kernel values evaluated on the fly
// instead of streamed: the same cluster pairs, bit masks, lane/warp mapping and sum
// order as pair_spmv_kernel, the table in shared memory.  Per pair the offset of the
// cluster centres under the minimum image comes from the mask pass; when
// rc + 2 (e_I + e_J) < L/2 along every axis (e the clusters' half extents) every
// in-range bead pair's separation is the plain difference of the bead offsets (a bead
// lies within e of its centre, so that difference is within rc + 2 (e_I + e_J) of zero
// and no other image can be nearer), otherwise each separation gets its own minimum
// image.
template <int W>
__global__ void __launch_bounds__(W * 32, 6) pair_otf32_kernel(const long long *__restrict__ head,
                                                               const int *__restrict__ count,
                                                               const int *__restrict__ pair_j,
                                                               const int *__restrict__ members,
                                                               const unsigned *__restrict__ masks,
                                                               const float4 *__restrict__ boff,
                                                               const float4 *__restrict__ pshift, RSBuild c,
                                                               const float2 *__restrict__ tab, float scale,
                                                               const float *__restrict__ qc,
                                                               const float *__restrict__ q,
                                                               const float *__restrict__ phik, double selfc,
                                                               const double *__restrict__ phi_body,
                                                               const uint32_t *__restrict__ body,
                                                               double *__restrict__ out) {
    extern __shared__ float2 stab[];
    __shared__ float part[W][CS];
    for (int k = threadIdx.x; k <= c.ntab; k += W * 32) stab[k] = tab[k];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int I = blockIdx.x;
    const float4 oi = boff[I * CS + lane];
    const long long h0 = head[I];
    const int n = count[I];
    const float dr = (float)c.dr, inv_dr = (float)c.inv_dr;
    const float3 L32 = make_float3((float)c.L[0], (float)c.L[1], (float)c.L[2]);
    const float3 Li32 = make_float3((float)c.Linv[0], (float)c.Linv[1], (float)c.Linv[2]);
    __syncthreads();
    float y = 0.f;
    for (int k = w; k < n; k += W) {
        const long long p = h0 + k;
        const int J = pair_j[p];
        const unsigned m = masks[p * CS + lane];
        const float4 oj = boff[J * CS + lane];
        const float qj = qc[J * CS + lane];
        const float4 sh = pshift[p];
        const bool direct = sh.w != 0.f;
        const float ax = oi.x - sh.x, ay = oi.y - sh.y, az = oi.z - sh.z;
        const unsigned steps = __reduce_max_sync(0xffffffffu, (unsigned)__popc(m));
        unsigned mm = m;
        if (direct) {
            for (unsigned t = 0; t < steps; ++t) {
                const bool has = mm != 0;
                const int j = has ? __ffs(mm) - 1 : 0;
                mm &= mm - 1;
                const float bx = __shfl_sync(0xffffffffu, oj.x, j);
                const float by = __shfl_sync(0xffffffffu, oj.y, j);
                const float bz = __shfl_sync(0xffffffffu, oj.z, j);
                const float qq = __shfl_sync(0xffffffffu, qj, j);
                if (has) {
                    const float dx = ax - bx, dy = ay - by, dz = az - bz;
                    y = fmaf(table_lerp32(stab, dx * dx + dy * dy + dz * dz, c.ntab, scale, dr, inv_dr), qq, y);
                }
            }
        } else {
            for (unsigned t = 0; t < steps; ++t) {
                const bool has = mm != 0;
                const int j = has ? __ffs(mm) - 1 : 0;
                mm &= mm - 1;
                const float bx = __shfl_sync(0xffffffffu, oj.x, j);
                const float by = __shfl_sync(0xffffffffu, oj.y, j);
                const float bz = __shfl_sync(0xffffffffu, oj.z, j);
                const float qq = __shfl_sync(0xffffffffu, qj, j);
                if (has) {
                    float dx = ax - bx, dy = ay - by, dz = az - bz;
                    dx -= L32.x * rintf(dx * Li32.x);
                    dy -= L32.y * rintf(dy * Li32.y);
                    dz -= L32.z * rintf(dz * Li32.z);
                    y = fmaf(table_lerp32(stab, dx * dx + dy * dy + dz * dz, c.ntab, scale, dr, inv_dr), qq, y);
                }
            }
        }
    }
    part[w][lane] = y;
    __syncthreads();
    if (w == 0) {
        float tot = 0.f;
#pragma unroll
        for (int v = 0; v < W; ++v) tot += part[v][lane];
        const int bi = members[I * CS + lane];
        if (bi >= 0) {
            const double total = (double)phik[bi] + selfc * (double)q[bi] + (double)tot;
            out[bi] = phi_body ? phi_body[body[bi]] - total : total;
        }
    }
}

// The FP64 product with the values evaluated on the fly: the arithmetic of
// pair_values_kernel (FP64 minimum image, reciprocal square root by Newton steps, the
// FP64 table lerp) and the sum order of pair_spmv_kernel, so the result equals the
// streamed FP64 product bit for bit.
template <int W>
__global__ void __launch_bounds__(W * 32) pair_otf64_kernel(const long long *__restrict__ head,
                                                            const int *__restrict__ count,
                                                            const int *__restrict__ pair_j,
                                                            const int *__restrict__ members,
                                                            const unsigned *__restrict__ masks,
                                                            const double4 *__restrict__ pos,
                                                            const double2 *__restrict__ tab, RSBuild c,
                                                            const double *__restrict__ qc,
                                                            const double *__restrict__ q,
                                                            const double *__restrict__ phik, double selfc,
                                                            const double *__restrict__ phi_body,
                                                            const uint32_t *__restrict__ body,
                                                            double *__restrict__ out) {
    __shared__ double part[W][CS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int I = blockIdx.x;
    const int bi = members[I * CS + lane];
    const double4 pi = bi >= 0 ? pos[bi] : make_double4(0, 0, 0, 0);
    const long long h0 = head[I];
    const int n = count[I];
    double y = 0.0;
    for (int k = w; k < n; k += W) {
        const long long p = h0 + k;
        const int J = pair_j[p];
        const unsigned m = masks[p * CS + lane];
        const int bj = members[J * CS + lane];
        const double4 pjl = bj >= 0 ? pos[bj] : make_double4(0, 0, 0, 0);
        const double qjl = qc[J * CS + lane];
        const unsigned steps = __reduce_max_sync(0xffffffffu, (unsigned)__popc(m));
        unsigned mm = m;
        for (unsigned t = 0; t < steps; ++t) {
            const bool has = mm != 0;
            const int j = has ? __ffs(mm) - 1 : 0;
            mm &= mm - 1;
            const double xj = __shfl_sync(0xffffffffu, pjl.x, j);
            const double yj = __shfl_sync(0xffffffffu, pjl.y, j);
            const double zj = __shfl_sync(0xffffffffu, pjl.z, j);
            const double qj = __shfl_sync(0xffffffffu, qjl, j);
            if (has) {
                const double dx = mimg(pi.x - xj, c.L[0], c.Linv[0]);
                const double dy = mimg(pi.y - yj, c.L[1], c.Linv[1]);
                const double dz = mimg(pi.z - zj, c.L[2], c.Linv[2]);
                const double d2 = dx * dx + dy * dy + dz * dz;
                y += table_lerp64(tab, c, d2 * rsqrt64(d2)) * qj;
            }
        }
    }
    part[w][lane] = y;
    __syncthreads();
    if (w == 0 && bi >= 0) {
        double tot = 0.0;
#pragma unroll
        for (int v = 0; v < W; ++v) tot += part[v][lane];
        const double total = phik[bi] + selfc * q[bi] + tot;
        out[bi] = phi_body ? phi_body[body[bi]] - total : total;
    }
}

// Real-space forces over the cluster pairs, on the fly in FP64: F_i += -T'(d) q_i q_j
// r_ij / d (ConductorRigid.cu:637-654); every ordered pair (I, J) is in the list.  One
// CTA per cluster I: warp w takes I's pairs w, w+W, ..., lane i accumulates bead i's
// force over the set bits of its mask rows, and the W partial forces are added in warp
// order and written once (no atomics, the same result on every run).
template <int W>
__global__ void __launch_bounds__(W * 32) pair_force_kernel(const long long *__restrict__ head,
                                                            const int *__restrict__ count,
                                                            const int *__restrict__ pair_j,
                                                            const int *__restrict__ members,
                                                            const unsigned *__restrict__ masks,
                                                            const double4 *__restrict__ pos,
                                                            const double *__restrict__ q,
                                                            const double2 *__restrict__ tab, RSBuild c,
                                                            double *__restrict__ F) {
    __shared__ double part[W][3][CS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int I = blockIdx.x;
    const int bi = members[I * CS + lane];
    const double4 pi = bi >= 0 ? pos[bi] : make_double4(0, 0, 0, 0);
    const double qi = bi >= 0 ? q[bi] : 0.0;
    double fi[3] = {0, 0, 0};
    const long long h0 = head[I];
    const int n = count[I];
    for (int k = w; k < n; k += W) {
        const long long p = h0 + k;
        const int J = pair_j[p];
        const unsigned m = masks[p * CS + lane];
        const int bj = members[J * CS + lane];
        const double4 pjl = bj >= 0 ? pos[bj] : make_double4(0, 0, 0, 0);
        const double qjl = bj >= 0 ? q[bj] : 0.0;
        // lane i walks its own set bits in ascending order (the in-range test of
        // pair_mask_kernel), the warp as many steps as its longest row
        const unsigned steps = __reduce_max_sync(0xffffffffu, (unsigned)__popc(m));
        unsigned mm = m;
        for (unsigned t = 0; t < steps; ++t) {
            const bool has = mm != 0;
            const int j = has ? __ffs(mm) - 1 : 0;
            mm &= mm - 1;
            const double xj = __shfl_sync(0xffffffffu, pjl.x, j);
            const double yj = __shfl_sync(0xffffffffu, pjl.y, j);
            const double zj = __shfl_sync(0xffffffffu, pjl.z, j);
            const double qj = __shfl_sync(0xffffffffu, qjl, j);
            if (has) {
                const double dx = mimg(pi.x - xj, c.L[0], c.Linv[0]);
                const double dy = mimg(pi.y - yj, c.L[1], c.Linv[1]);
                const double dz = mimg(pi.z - zj, c.L[2], c.Linv[2]);
                const double d2 = dx * dx + dy * dy + dz * dz;
                const double inv_d = rsqrt64(d2);
                const double a = -table_lerp64(tab, c, d2 * inv_d) * qi * qj * inv_d;
                fi[0] += a * dx;
                fi[1] += a * dy;
                fi[2] += a * dz;
            }
        }
    }
    for (int e = 0; e < 3; ++e) part[w][e][lane] = fi[e];
    __syncthreads();
    if (w == 0 && bi >= 0) {
        for (int e = 0; e < 3; ++e) {
            double t = 0.0;
#pragma unroll
            for (int v = 0; v < W; ++v) t += part[v][e][lane];
            F[3 * (size_t)bi + e] = t;
        }
    }
}

// Real-space virial -dU_real/de_ab = 1/2 sum_{i != j} r_ij,a F_ij,b with the pair force
// F_ij = -T'(d) q_i q_j r_ij / d of pair_force_kernel (the same pairs, gradient table and
// FP64 arithmetic).  One CTA per cluster I writes its six components (xx, xy, xz, yy,
// yz, zz) to partial[I][6]; the host adds the clusters in order.
template <int W>
__global__ void __launch_bounds__(W * 32) pair_virial_kernel(const long long *__restrict__ head,
                                                             const int *__restrict__ count,
                                                             const int *__restrict__ pair_j,
                                                             const int *__restrict__ members,
                                                             const unsigned *__restrict__ masks,
                                                             const double4 *__restrict__ pos,
                                                             const double *__restrict__ q,
                                                             const double2 *__restrict__ tab, RSBuild c,
                                                             double *__restrict__ partial) {
    __shared__ double red[W][6];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int I = blockIdx.x;
    const int bi = members[I * CS + lane];
    const double4 pi = bi >= 0 ? pos[bi] : make_double4(0, 0, 0, 0);
    const double qi = bi >= 0 ? q[bi] : 0.0;
    double v[6] = {0, 0, 0, 0, 0, 0};
    const long long h0 = head[I];
    const int n = count[I];
    for (int k = w; k < n; k += W) {
        const long long p = h0 + k;
        const int J = pair_j[p];
        const unsigned m = masks[p * CS + lane];
        const int bj = members[J * CS + lane];
        const double4 pjl = bj >= 0 ? pos[bj] : make_double4(0, 0, 0, 0);
        const double qjl = bj >= 0 ? q[bj] : 0.0;
        const unsigned steps = __reduce_max_sync(0xffffffffu, (unsigned)__popc(m));
        unsigned mm = m;
        for (unsigned t = 0; t < steps; ++t) {
            const bool has = mm != 0;
            const int j = has ? __ffs(mm) - 1 : 0;
            mm &= mm - 1;
            const double xj = __shfl_sync(0xffffffffu, pjl.x, j);
            const double yj = __shfl_sync(0xffffffffu, pjl.y, j);
            const double zj = __shfl_sync(0xffffffffu, pjl.z, j);
            const double qj = __shfl_sync(0xffffffffu, qjl, j);
            if (has) {
                const double dx = mimg(pi.x - xj, c.L[0], c.Linv[0]);
                const double dy = mimg(pi.y - yj, c.L[1], c.Linv[1]);
                const double dz = mimg(pi.z - zj, c.L[2], c.Linv[2]);
                const double d2 = dx * dx + dy * dy + dz * dz;
                const double inv_d = rsqrt64(d2);
                const double a = -table_lerp64(tab, c, d2 * inv_d) * qi * qj * inv_d;
                v[0] += a * dx * dx;
                v[1] += a * dx * dy;
                v[2] += a * dx * dz;
                v[3] += a * dy * dy;
                v[4] += a * dy * dz;
                v[5] += a * dz * dz;
            }
        }
    }
    for (int e = 0; e < 6; ++e) {
        double t = v[e];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) red[w][e] = t;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double t = 0.0;
#pragma unroll
        for (int u = 0; u < W; ++u) t += red[u][threadIdx.x];
        partial[(size_t)I * 6 + threadIdx.x] = 0.5 * t;
    }
}

// force_i = wave force_i + q_i E0 + real-space force_i
template <typename R>
__global__ void force_combine_kernel(int N, const R *__restrict__ fk, const double *__restrict__ q, double Ex,
                                     double Ey, double Ez, const double *__restrict__ freal, double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double qi = q[i];
    out[3 * (size_t)i + 0] = (double)fk[3 * (size_t)i + 0] + qi * Ex + freal[3 * (size_t)i + 0];
    out[3 * (size_t)i + 1] = (double)fk[3 * (size_t)i + 1] + qi * Ey + freal[3 * (size_t)i + 1];
    out[3 * (size_t)i + 2] = (double)fk[3 * (size_t)i + 2] + qi * Ez + freal[3 * (size_t)i + 2];
}

RSBuild rs_build(const cr_handle *h) {
    RSBuild c;
    for (int d = 0; d < 3; ++d) {
        c.L[d] = h->L[d];
        c.Linv[d] = 1.0 / h->L[d];
    }
    c.rc = h->d.rcut;
    c.rc2 = h->d.rcut * h->d.rcut;
    c.rmin2 = h->d.dr * h->d.dr;
    c.dr = h->d.dr;
    c.inv_dr = 1.0 / h->d.dr;
    c.ntab = h->d.n_table;
    c.scale = h->d.n_table / (h->d.rcut - h->d.dr);
    return c;
}

template <typename R> R *acc_of(RealSpace &r);
template <> float *acc_of<float>(RealSpace &r) { return r.acc32; }
template <> double *acc_of<double>(RealSpace &r) { return r.acc64; }
template <typename R> R *&blocks_of(RealSpace &r);
template <> float *&blocks_of<float>(RealSpace &r) { return r.vals32; }
template <> double *&blocks_of<double>(RealSpace &r) { return r.vals64; }
template <typename R> bool &valid_of(RealSpace &r);
template <> bool &valid_of<float>(RealSpace &r) { return r.valid32; }
template <> bool &valid_of<double>(RealSpace &r) { return r.valid64; }
template <typename R> long long &cap_of(RealSpace &r);
template <> long long &cap_of<float>(RealSpace &r) { return r.blocks32_cap; }
template <> long long &cap_of<double>(RealSpace &r) { return r.blocks64_cap; }

template <typename R> int realspace_reserve(cr_handle *h) {
    RealSpace &r = h->rs;
    const long long need = std::max(r.nnz, 1LL);
    if (need > cap_of<R>(r)) {
        const long long cap = need + need / 8;
        CR_TRY(dalloc(h, &blocks_of<R>(r), (size_t)cap));
        cap_of<R>(r) = cap;
    }
    return CR_OK;
}

// Packed values of precision R for the current cluster pairs (once per solve).  A solve
// that runs an FP32 operator also needs FP64 values (its true residuals), so in those
// modes the first request builds both in one pass.
// Shared memory of the FP32 table (value, next value) of the on-the-fly product; tables
// beyond the default 48 KB of dynamic shared memory (rc > 6.1) keep the stored values.
size_t onfly32_smem(const cr_handle *h) { return (size_t)(h->d.n_table + 1) * sizeof(float2); }

template <typename R> bool onfly(const cr_handle *h) {
    if (sizeof(R) == 4) return (h->rs_onfly & CR_REALSPACE_ONFLY32) && onfly32_smem(h) <= 48 * 1024;
    return h->rs_onfly & CR_REALSPACE_ONFLY64;
}

template <typename R> int realspace_blocks(cr_handle *h) {
    RealSpace &r = h->rs;
    if (valid_of<R>(r) || h->N == 0 || onfly<R>(h)) return CR_OK;
    if (h->user.precision != CR_FP64 && !r.valid32 && !r.valid64 && !onfly<float>(h) && !onfly<double>(h)) {
        CR_TRY(realspace_reserve<float>(h));
        CR_TRY(realspace_reserve<double>(h));
        pair_values_kernel<float, double><<<blocks_for(r.npairs * 32, 256), 256, 0, h->stream>>>(
            r.npairs, r.pair_i, r.pair_j, r.members, h->m64.pos, h->m64.phiq, rs_build(h), r.masks, r.voff,
            r.nnz_pair, r.vals32, r.vals64);
        CR_LAUNCH(h, "pair_values_kernel");
        r.valid32 = r.valid64 = true;
        return CR_OK;
    }
    CR_TRY(realspace_reserve<R>(h));
    pair_values_kernel<R><<<blocks_for(r.npairs * 32, 256), 256, 0, h->stream>>>(
        r.npairs, r.pair_i, r.pair_j, r.members, h->m64.pos, h->m64.phiq, rs_build(h), r.masks, r.voff, r.nnz_pair,
        blocks_of<R>(r));
    CR_LAUNCH(h, "pair_values_kernel");
    valid_of<R>(r) = true;
    return CR_OK;
}

}  // namespace

// Build the stored values of the given operator precision for the current geometry now
// (the operator otherwise builds them on its first application).
int realspace_prepare(cr_handle *h, int precision) {
    return precision == CR_FP64 ? realspace_blocks<double>(h) : realspace_blocks<float>(h);
}

void realspace_free(cr_handle *h) {
    RealSpace &r = h->rs;
    dfree(&r.members);
    dfree(&r.centre);
    dfree(&r.extent);
    dfree(&r.count);
    dfree(&r.head);
    dfree(&r.pair_i);
    dfree(&r.pair_j);
    dfree(&r.vals32);
    dfree(&r.vals64);
    dfree(&r.masks);
    dfree(&r.nnz_pair);
    dfree(&r.voff);
    dfree(&r.acc32);
    dfree(&r.acc64);
    dfree(&r.freal);
    dfree(&r.bits);
    dfree(&r.boff);
    dfree(&r.pshift);
    r.pair_cap = 0;
    r.nnz = 0;
    r.blocks32_cap = r.blocks64_cap = 0;
    r.npairs = 0;
    r.valid32 = r.valid64 = false;
}

int realspace_alloc(cr_handle *h) {
    RealSpace &r = h->rs;
    realspace_free(h);

    r.nclus = (h->N + CS - 1) / CS;
    const size_t nc = (size_t)std::max(r.nclus, 1);
    CR_TRY(dalloc(h, &r.members, nc * CS));
    CR_TRY(dalloc(h, &r.centre, nc));
    CR_TRY(dalloc(h, &r.extent, nc));
    CR_TRY(dalloc(h, &r.count, nc));
    CR_TRY(dalloc(h, &r.head, nc));
    CR_TRY(dalloc(h, &r.sorted, (size_t)std::max(h->N, 1)));
    CR_TRY(dalloc(h, &r.acc32, nc * CS));
    CR_TRY(dalloc(h, &r.acc64, nc * CS));
    CR_TRY(dalloc(h, &r.freal, 3 * (size_t)std::max(h->N, 1)));
    CR_TRY(dalloc(h, &r.bits, 1));
    CR_TRY(dalloc(h, &r.boff, nc * CS));
    return CR_OK;
}

// Clusters and cluster pairs of the current positions; blocks are filled on first
// use per precision.
int realspace_build(cr_handle *h) {
    RealSpace &r = h->rs;
    const int N = h->N;
    r.valid32 = r.valid64 = false;
    if (N == 0) return CR_OK;
    cudaStream_t s = h->stream;
    const RSBuild c = rs_build(h);
    morton_kernel<<<blocks_for(N, 256), 256, 0, s>>>(N, h->m64.pos, h->L[0], h->L[1], h->L[2], h->d_keys,
                                                     h->d_vals_alt);
    CR_LAUNCH(h, "morton_kernel");
    size_t bytes = h->sort_tmp_bytes;
    CR_CUDA(h, cub::DeviceRadixSort::SortPairs(h->d_sort_tmp, bytes, h->d_keys, h->d_keys_alt, h->d_vals_alt,
                                               r.sorted, N, 0, 30, s));
    const int nb = blocks_for((long)r.nclus * 32, 256);
    cluster_kernel<<<nb, 256, 0, s>>>(N, r.nclus, r.sorted, h->m64.pos, c, r.members, r.centre, r.extent);
    CR_LAUNCH(h, "cluster_kernel");
    cluster_offsets_kernel<<<nb, 256, 0, s>>>(r.nclus * CS, r.members, h->m64.pos, r.centre, c, r.boff);
    CR_LAUNCH(h, "cluster_offsets_kernel");
    pair_search_kernel<false><<<nb, 256, 0, s>>>(r.nclus, r.centre, r.extent, c, r.count, nullptr, nullptr);
    CR_LAUNCH(h, "pair_search_kernel");
    bytes = h->sort_tmp_bytes;
    CR_CUDA(h, cub::DeviceScan::ExclusiveSum(h->d_sort_tmp, bytes, r.count, r.head, r.nclus, s));
    long long last_head = 0;
    int last_count = 0;
    CR_CUDA(h, cudaMemcpyAsync(&last_head, r.head + r.nclus - 1, sizeof(long long), cudaMemcpyDeviceToHost, s));
    CR_CUDA(h, cudaMemcpyAsync(&last_count, r.count + r.nclus - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    CR_CUDA(h, cudaStreamSynchronize(s));
    r.npairs = last_head + last_count;
    if (r.npairs > r.pair_cap) {
        const long long cap = r.npairs + r.npairs / 8 + 64;
        CR_TRY(dalloc(h, &r.pair_i, (size_t)cap));
        CR_TRY(dalloc(h, &r.pair_j, (size_t)cap));
        CR_TRY(dalloc(h, &r.masks, (size_t)cap * CS));
        CR_TRY(dalloc(h, &r.nnz_pair, (size_t)cap));
        CR_TRY(dalloc(h, &r.voff, (size_t)cap));
        CR_TRY(dalloc(h, &r.pshift, (size_t)cap));
        r.pair_cap = cap;
        // scan scratch for npairs entries
        size_t b = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, b, r.nnz_pair, r.voff, (int)cap);
        if (b + 256 > h->sort_tmp_bytes) {
            dfree(reinterpret_cast<char **>(&h->d_sort_tmp));
            CR_TRY(dalloc(h, reinterpret_cast<char **>(&h->d_sort_tmp), b + 256));
            h->sort_tmp_bytes = b + 256;
        }
    }
    pair_search_kernel<true><<<nb, 256, 0, s>>>(r.nclus, r.centre, r.extent, c, r.count, r.head, r.pair_j);
    CR_LAUNCH(h, "pair_search_kernel");
    pair_owner_kernel<<<r.nclus, 128, 0, s>>>(r.nclus, r.head, r.count, r.pair_i);
    CR_LAUNCH(h, "pair_owner_kernel");
    const int pb = blocks_for(r.npairs * 32, 256);
    CR_CUDA(h, cudaMemsetAsync(r.bits, 0, sizeof(unsigned long long), s));
    {
        const double Lmax = std::max(h->L[0], std::max(h->L[1], h->L[2]));
        const float band = (float)(1e-5 * c.rc * Lmax + 4e-6 * c.rc2);
        const float low = (float)(2.0 * c.rmin2) + band;
        pair_mask_kernel<<<pb, 256, 0, s>>>(r.npairs, r.pair_i, r.pair_j, r.members, h->m64.pos, h->m32.pos, c,
                                            make_float3((float)h->L[0], (float)h->L[1], (float)h->L[2]),
                                            make_float3((float)(1.0 / h->L[0]), (float)(1.0 / h->L[1]),
                                                        (float)(1.0 / h->L[2])),
                                            (float)c.rc2, band, low, r.masks, r.nnz_pair, r.bits, r.centre,
                                            r.extent, r.pshift);
    }
    CR_LAUNCH(h, "pair_mask_kernel");
    bytes = h->sort_tmp_bytes;
    CR_CUDA(h, cub::DeviceScan::ExclusiveSum(h->d_sort_tmp, bytes, r.nnz_pair, r.voff, (int)r.npairs, s));
    long long last_off = 0;
    int last_nnz = 0;
    unsigned long long nbits = 0;
    CR_CUDA(h, cudaMemcpyAsync(&nbits, r.bits, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CR_CUDA(h, cudaMemcpyAsync(&last_off, r.voff + r.npairs - 1, sizeof(long long), cudaMemcpyDeviceToHost, s));
    CR_CUDA(h, cudaMemcpyAsync(&last_nnz, r.nnz_pair + r.npairs - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    CR_CUDA(h, cudaStreamSynchronize(s));
    r.nnz = last_off + last_nnz;
    r.npairs_beads = (long long)nbits;
    // interacting (directed) bead pairs of one real-space application
    h->geo.nl_total = r.npairs_beads;
    return CR_OK;
}

template <typename R> int real_space_apply(cr_handle *h, MeshBuffers<R> &m, const double *phi_body, double *out) {
    const int N = h->N;
    if (N == 0) return CR_OK;
    RealSpace &r = h->rs;
    {
        ProfScope pb(h, PROF_GEOMETRY);
        CR_TRY(realspace_blocks<R>(h));
    }
    ProfScope ps(h, PROF_REAL);
    R *qc = acc_of<R>(r);
    gather_cluster_kernel<R><<<blocks_for((long)r.nclus * CS, 256), 256, 0, h->stream>>>(r.nclus * CS, r.members,
                                                                                         m.q, qc);
    CR_LAUNCH(h, "gather_cluster_kernel");
    constexpr int W = kSpmvWarps;
    if (onfly<R>(h)) {
        if constexpr (sizeof(R) == 4) {
            pair_otf32_kernel<W><<<r.nclus, W * 32, onfly32_smem(h), h->stream>>>(
                r.head, r.count, r.pair_j, r.members, r.masks, r.boff, r.pshift, rs_build(h), h->m32.phiq,
                (float)(h->d.n_table / (h->d.rcut - h->d.dr)), qc, m.q, m.phi, h->d.selfcoeff, phi_body, h->d_body,
                out);
            CR_LAUNCH(h, "pair_otf32_kernel");
        } else {
            pair_otf64_kernel<W><<<r.nclus, W * 32, 0, h->stream>>>(r.head, r.count, r.pair_j, r.members, r.masks,
                                                                    h->m64.pos, h->m64.phiq, rs_build(h), qc, m.q,
                                                                    m.phi, h->d.selfcoeff, phi_body, h->d_body, out);
            CR_LAUNCH(h, "pair_otf64_kernel");
        }
        return CR_OK;
    }
    pair_spmv_kernel<R, W, 16><<<r.nclus, W * 32, 0, h->stream>>>(
        r.nclus, r.head, r.count, r.pair_j, r.members, r.masks, r.voff, r.nnz_pair, blocks_of<R>(r), qc, m.q, m.phi,
        h->d.selfcoeff, phi_body, h->d_body, out);
    CR_LAUNCH(h, "pair_spmv_kernel");
    return CR_OK;
}

template <typename R> int real_space_force(cr_handle *h, MeshBuffers<R> &m, const double *q64, double *force_out) {
    const int N = h->N;
    if (N == 0) return CR_OK;
    RealSpace &r = h->rs;
    ProfScope ps(h, PROF_REAL_FORCE);
    CR_CUDA(h, cudaMemsetAsync(r.freal, 0, 3 * (size_t)N * sizeof(double), h->stream));  // beads without pairs
    pair_force_kernel<kSpmvWarps><<<r.nclus, kSpmvWarps * 32, 0, h->stream>>>(
        r.head, r.count, r.pair_j, r.members, r.masks, h->m64.pos, q64, h->m64.gradphiq, rs_build(h), r.freal);
    CR_LAUNCH(h, "pair_force_kernel");
    force_combine_kernel<R><<<blocks_for(N, 256), 256, 0, h->stream>>>(N, m.force, q64, h->field[0], h->field[1],
                                                                       h->field[2], r.freal, force_out);
    CR_LAUNCH(h, "force_combine_kernel");
    return CR_OK;
}

int real_space_virial(cr_handle *h, const double *q64, double *out) {
    for (int e = 0; e < 6; ++e) out[e] = 0.0;
    if (h->N == 0) return CR_OK;
    RealSpace &r = h->rs;
    std::vector<double> part((size_t)r.nclus * 6);
    double *d_part = nullptr;
    CR_TRY(dalloc(h, &d_part, part.size()));
    pair_virial_kernel<kSpmvWarps><<<r.nclus, kSpmvWarps * 32, 0, h->stream>>>(
        r.head, r.count, r.pair_j, r.members, r.masks, h->m64.pos, q64, h->m64.gradphiq, rs_build(h), d_part);
    int st = check_cuda(h, cudaGetLastError(), "pair_virial_kernel");
    if (st == CR_OK) {
        ++h->launches;
        st = check_cuda(h, cudaMemcpyAsync(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                           h->stream), "real-space virial partials");
    }
    if (st == CR_OK) st = check_cuda(h, cudaStreamSynchronize(h->stream), "real-space virial");
    dfree(&d_part);
    if (st != CR_OK) return st;
    for (int I = 0; I < r.nclus; ++I)
        for (int e = 0; e < 6; ++e) out[e] += part[(size_t)I * 6 + e];
    return CR_OK;
}

template int real_space_apply<float>(cr_handle *, MeshBuffers<float> &, const double *, double *);
template int real_space_apply<double>(cr_handle *, MeshBuffers<double> &, const double *, double *);
template int real_space_force<float>(cr_handle *, MeshBuffers<float> &, const double *, double *);
template int real_space_force<double>(cr_handle *, MeshBuffers<double> &, const double *, double *);

}  // namespace cr
