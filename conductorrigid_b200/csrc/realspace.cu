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
//    pair are stored in row groups: rows in groups of 8 lanes, each group padded with
//    zeros to its longest row, the k-th value of a row in slot k of its group (8
//    consecutive values, one 32-byte sector in FP32), so that every load of a warp is
//    four whole sectors;
//  * the product y_I = sum_J B_IJ x_J, the pairs of cluster I split over the warps of
//    one CTA: lane i takes the k-th set bit j of its row (from the highest column
//    down), multiplies the k-th value by x_J[j] fetched with a warp shuffle; the
//    partial sums are added in warp order, so there are no atomics and the sum order
//    is fixed.  An alternative product streams the values through shared memory with
//    bulk copies (pair_stream_kernel, CR_REALSPACE_STREAM).
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

#ifndef CR_RS_GROUP
#define CR_RS_GROUP 8
#endif
// Stored layout of one cluster pair's values: its 32 rows in groups of RG lanes; group g
// holds rows_g slots (its longest row) of RG values, the k-th value of row i at
// off_g + k*RG + (i mod RG), the groups one after the other.  RG = 32 is the plain
// lane-interleaved layout (one 128-byte line per FP32 slot); smaller groups pad less.
constexpr int RG = CR_RS_GROUP;
static_assert(RG == 8 || RG == 16 || RG == 32, "row group of 8, 16 or 32 lanes");

struct RowGroup {
    int rows;   // slots of this lane's group
    int off;    // position of this lane's slot 0 within the pair's values
    int total;  // stored slots of the pair
};

__device__ __forceinline__ RowGroup row_group(unsigned m, int lane) {
    if (RG == CS) {
        const int rows = (int)__reduce_max_sync(0xffffffffu, (unsigned)__popc(m));
        return RowGroup{rows, lane, rows * CS};
    }
    int rg = __popc(m);
#pragma unroll
    for (int o = 1; o < RG; o <<= 1) rg = max(rg, __shfl_xor_sync(0xffffffffu, rg, o));
    RowGroup g{rg, lane & (RG - 1), 0};
#pragma unroll
    for (int k = 0; k < CS / RG; ++k) {
        const int sz = __shfl_sync(0xffffffffu, rg, k * RG) * RG;
        if (k < lane / RG) g.off += sz;
        g.total += sz;
    }
    return g;
}

// Bit masks of the in-range bead pairs of every cluster pair (row i = bead i of I,
// bit j = bead j of J) and the stored slots of the pair (per group of RG rows, RG times
// the group's longest row).
// The test runs in FP32 on the beads' offsets from their cluster centres and the centres'
// minimum-image offset (for cluster pairs whose bead separations need no further image,
// almost all of them), otherwise on the FP32 copies of the positions; only a pair whose
// FP32 squared distance lies within `band` of rc^2 (or below 2 dr^2 + band) is decided
// again in FP64, exactly as the oracle decides it.  `band` is ten times a bound on the
// FP32 error of d^2 for |d| <= rc in a box of edge L (positions rounded to FP32: |error of
// dx| <= 2e-7 L; the offsets, a few units long, are rounded far more finely), so the masks
// equal the FP64 ones bit for bit.
__global__ void pair_mask_kernel(long long npairs, const int *__restrict__ pair_i, const int *__restrict__ pair_j,
                                 const int *__restrict__ members, const double4 *__restrict__ pos,
                                 const float4 *__restrict__ pos32, RSBuild c, float3 L32, float3 Linv32, float rc2,
                                 float band, float low, unsigned *__restrict__ masks, int *__restrict__ nnz,
                                 unsigned long long *__restrict__ bits, const double4 *__restrict__ centre,
                                 const double4 *__restrict__ extent, const float4 *__restrict__ boff,
                                 float4 *__restrict__ pshift) {
    const long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= npairs) return;
    const int I = pair_i[p], J = pair_j[p];
    const int bi = members[I * CS + lane];
    const int bj = members[J * CS + lane];
    // offset of the cluster centres under the minimum image, and whether the bead offsets
    // then need no further image: rc + 2 (e_I + e_J) < L/2 along every axis (a bead lies
    // within e of its centre, so no other image of a pair within rc can be nearer)
    const double4 cI = centre[I], cJ = centre[J], eI = extent[I], eJ = extent[J];
    const bool direct = c.rc + 2.0 * (eI.x + eJ.x) < 0.5 * c.L[0] - 1e-3 &&
                        c.rc + 2.0 * (eI.y + eJ.y) < 0.5 * c.L[1] - 1e-3 &&
                        c.rc + 2.0 * (eI.z + eJ.z) < 0.5 * c.L[2] - 1e-3;
    const float4 sh = make_float4((float)mimg(cJ.x - cI.x, c.L[0], c.Linv[0]), (float)mimg(cJ.y - cI.y, c.L[1], c.Linv[1]),
                                  (float)mimg(cJ.z - cI.z, c.L[2], c.Linv[2]), direct ? 1.f : 0.f);
    unsigned m = 0;
    if (direct) {
        // separations from the FP32 offsets of the beads from their cluster centres: d =
        // (o_i - shift) - o_j.  Padding beads sit at +-1e30, so every separation with one
        // of them overflows to infinity and fails the test without a check per bead.
        const float4 oi = boff[I * CS + lane], oj = boff[J * CS + lane];
        const float ax = bi >= 0 ? oi.x - sh.x : 1e30f, ay = bi >= 0 ? oi.y - sh.y : 1e30f,
                    az = bi >= 0 ? oi.z - sh.z : 1e30f;
        const float jx = bj >= 0 ? oj.x : -1e30f, jy = bj >= 0 ? oj.y : -1e30f, jz = bj >= 0 ? oj.z : -1e30f;
#pragma unroll 8
        for (int j = 0; j < CS; ++j) {
            const float dx = ax - __shfl_sync(0xffffffffu, jx, j);
            const float dy = ay - __shfl_sync(0xffffffffu, jy, j);
            const float dz = az - __shfl_sync(0xffffffffu, jz, j);
            const float d2 = dx * dx + dy * dy + dz * dz;
            bool in;
            if (d2 > rc2 + band) {
                in = false;
            } else if (d2 < rc2 - band && d2 > low) {
                in = true;
            } else {  // near a boundary (both beads real): the FP64 decision of the oracle
                const double4 a = pos[bi], b = pos[members[J * CS + j]];
                const double e2 = dist2_exact(a, b, c);
                in = e2 < c.rc2 && e2 >= c.rmin2;
            }
            if (in) m |= 1u << j;
        }
    } else {
        const float4 pi = bi >= 0 ? pos32[bi] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 pjl = bj >= 0 ? pos32[bj] : make_float4(0.f, 0.f, 0.f, 0.f);
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
    }
    masks[p * CS + lane] = m;
    const int stored = row_group(m, lane).total;
    const int tot = (int)__reduce_add_sync(0xffffffffu, (unsigned)__popc(m));
    if (lane == 0) {
        nnz[p] = stored;
        atomicAdd(bits, (unsigned long long)tot);
        pshift[p] = sh;
    }
}

// The stored values of a row, and every product that must reproduce their sums, walk the
// row's set bits from the highest column down: the position of the highest set bit is
// one `bfind` (0xffffffff for an empty row, which a shuffle reads as lane 31 against a
// zero value), and clearing it is one mask of the bits below it (`bmsk.clamp` of width
// 0xffffffff keeps every bit, so an empty row stays empty).
__device__ __forceinline__ int top_bit(unsigned m) {
    int j;
    asm("bfind.u32 %0, %1;" : "=r"(j) : "r"(m));
    return j;
}
__device__ __forceinline__ unsigned below_bit(unsigned m, int j) {
    unsigned k;
    asm("bmsk.clamp.b32 %0, 0, %1;" : "=r"(k) : "r"(j));
    return m & k;
}

// Row i of the operator's top block from the real-space sum y_i: Phi_body(i) - (phik_i +
// self q_i + y_i), or the bare sum when phi_body is NULL.  With phik NULL only y_i is
// written: the wave-space part is then still being computed on another stream and
// rows_combine_kernel adds it afterwards, with the same arithmetic.
template <typename R>
__device__ __forceinline__ void write_row(double *__restrict__ out, int bi, double y, const R *__restrict__ phik,
                                          const R *__restrict__ q, double selfc, const double *__restrict__ phi_body,
                                          const uint32_t *__restrict__ body) {
    if (!phik) {
        out[bi] = y;
        return;
    }
    const double total = (double)phik[bi] + selfc * (double)q[bi] + y;
    out[bi] = phi_body ? phi_body[body[bi]] - total : total;
}

template <typename R>
__global__ void rows_combine_kernel(int N, const R *__restrict__ phik, const R *__restrict__ q, double selfc,
                                    const double *__restrict__ phi_body, const uint32_t *__restrict__ body,
                                    double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) write_row(out, i, out[i], phik, q, selfc, phi_body, body);
}

// Values T(d_ij) of the set mask bits in the operator precision, in the row-group
// layout: the k-th set bit of row i, counted from the highest column down, in slot k of
// the row, zeros after the row's last bit up to its group's longest row.
// With R2 = double (and R = float) one pass writes both precisions' values.
template <typename R, typename R2 = void>
__global__ void pair_values_kernel(long long npairs, const int *__restrict__ pair_i, const int *__restrict__ pair_j,
                                   const int *__restrict__ members, const double4 *__restrict__ pos,
                                   const double2 *__restrict__ tab, RSBuild c, const unsigned *__restrict__ masks,
                                   const long long *__restrict__ voff, R *__restrict__ vals,
                                   double *__restrict__ vals2 = nullptr) {
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
    const RowGroup g = row_group(m, lane);
    R *out = vals + voff[p] + g.off;
    double *out2 = BOTH ? vals2 + voff[p] + g.off : nullptr;
    // lane i walks its own set bits from the top (the k-th bit j at step k), fetching bead
    // j's position from lane j; lanes past their last bit write the zero padding of the slot
    const int rows = (int)__reduce_max_sync(0xffffffffu, (unsigned)g.rows);
    unsigned mm = m;
    for (int k = 0; k < rows; ++k) {
        const bool has = mm != 0;
        const int j = top_bit(mm) & 31;
        mm = below_bit(mm, j);
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
        if (k < g.rows) {
            out[(size_t)k * RG] = (R)t;
            if (BOTH) out2[(size_t)k * RG] = t;
        }
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
// bits of its mask row from the top, the k-th against the coalesced load of slot k, with
// x_J[j] from a shuffle (per slot: load, bfind, bmsk, and, shuffle, multiply-add).  Up to U slots are loaded before they are used; the next
// pair's metadata is fetched while the current one is summed.  The W partial sums are
// added in warp order, so the result does not depend on scheduling.
// FP32: six CTAs per SM (at most 40 registers; 48 warps of loads in flight, 0.864 ->
// 0.835 ms per application at 162k charges; 32 registers spill and lose it again).
// (cluster I: the body of pair_spmv_kernel and of its lockstep-batch form)
template <typename R, int W, int U>
__device__ __forceinline__ void pair_spmv_cluster(int I, const long long *__restrict__ head,
                                                  const int *__restrict__ count, const int *__restrict__ pair_j,
                                                  const int *__restrict__ members, const unsigned *__restrict__ masks,
                                                  const long long *__restrict__ voff, const int *__restrict__ slots,
                                                  const R *__restrict__ vals, const R *__restrict__ qc,
                                                  const R *__restrict__ q, const R *__restrict__ phik, double selfc,
                                                  const double *__restrict__ phi_body,
                                                  const uint32_t *__restrict__ body, double *__restrict__ out) {
    __shared__ R part[W][CS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    R yI = 0, yI2 = 0;  // FP32: odd slots into a second sum (half the dependent-add chain)
    const long long h0 = head[I];
    const int n = count[I];
    int J = 0;
    unsigned m0 = 0;
    long long off = 0;
    R xJ = 0;
    long long offn = 0;  // values offset and stored slots of the pair after the next one
    int sln = 0;
    if (w < n) {
        J = pair_j[h0 + w];
        m0 = masks[(h0 + w) * CS + lane];
        off = voff[h0 + w];
        xJ = qc[J * CS + lane];
    }
    if (w + W < n) {
        offn = voff[h0 + w + W];
        sln = slots[h0 + w + W];
    }
    for (int k = w; k < n; k += W) {
        unsigned m = m0;
        const RowGroup g = row_group(m, lane);
        const R *v = vals + off + g.off;
        const int rcur = RG == CS ? g.rows : (int)__reduce_max_sync(0xffffffffu, (unsigned)g.rows);
        const R xcur = xJ;
        if (k + W < n) {
            // the next pair's values into L2 while this pair is summed (one bulk prefetch;
            // offsets and sizes are multiples of 32 bytes)
            if (lane == 0 && sln > 0)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(vals + offn),
                             "r"((unsigned)(sln * sizeof(R)))
                             : "memory");
            const long long p1 = h0 + k + W;
            J = pair_j[p1];
            m0 = masks[p1 * CS + lane];
            off = offn;
            xJ = qc[J * CS + lane];
            if (k + 2 * W < n) {
                offn = voff[p1 + W];
                sln = slots[p1 + W];
            }
        }
        // slots past the end of a lane's row hold zeros and its walk then reads lane 31
        for (int base = 0; base < rcur; base += U) {
            R t[U];
#pragma unroll
            for (int u = 0; u < U; ++u) t[u] = base + u < g.rows ? __ldg(v + (size_t)(base + u) * RG) : (R)0;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = top_bit(m);
                m = below_bit(m, j);
                const R xj = __shfl_sync(0xffffffffu, xcur, j);
                if (sizeof(R) == 4 && (u & 1)) {
                    yI2 += t[u] * xj;
                } else {
                    yI += t[u] * xj;
                }
            }
        }
    }
    part[w][lane] = yI + yI2;
    __syncthreads();
    if (w == 0) {
        R tot = 0;
#pragma unroll
        for (int v = 0; v < W; ++v) tot += part[v][lane];
        const int bi = members[I * CS + lane];
        if (bi >= 0) {
            write_row(out, bi, (double)tot, phik, q, selfc, phi_body, body);
        }
    }
}

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
    pair_spmv_cluster<R, W, U>(blockIdx.x, head, count, pair_j, members, masks, voff, slots, vals, qc, q, phik, selfc,
                               phi_body, body, out);
}

// ---- streamed product: a bulk-copy producer warp per CTA ------------------------------
//
// The direct product above keeps at most U slots of loads in flight per warp, as many as
// its registers hold.  Here a CTA owns a contiguous range of clusters (balanced by
// stored bytes) and one producer thread streams the range's values through a ring of
// shared-memory stages with cp.async.bulk (no multicast), each stage's completion
// signalled on its mbarrier by the byte count; the consumer warps read the values from
// shared memory.  A stage holds one chunk: the pairs whose values start in one 8 KB
// window of the range, so a chunk never splits a pair and spans at most 8 KB plus one
// pair.  Every consumer warp waits for every chunk in order and releases it (one arrival
// per warp on the stage's empty barrier) once its later pairs all start in later chunks;
// the warp holding the oldest chunk never waits on another warp, so the ring always
// moves.  The pairs of a cluster go to the consumer warps in turn and each warp adds its
// partial sums of a cluster to the cluster's 32 sums with one coalesced atomic add
// (stream_finish_kernel then forms the rows and clears the sums).  Every wait is
// bounded: a wait that runs out (or finds that another warp's did) sets the abort flag
// and the error word; the consumers then skip the remaining pairs, and the producer
// stops issuing and, as always before it returns, waits for its copies in flight.
constexpr int kStreamStages = 4;
constexpr int kStreamChunk = 16384;  // bytes per stage
constexpr int kStreamShift = 13;     // 8 KB windows
constexpr int kStreamWarps = 8;      // consumer warps per CTA, plus one producer warp
constexpr int kStreamCtasPerSm = 3;
static_assert((1 << kStreamShift) + CS * CS * 8 <= kStreamChunk, "a stage holds a window plus one FP64 pair");
constexpr long long kDrainLimit = 1LL << 33;  // cycles; copies in flight always complete

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool bar_ready(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Wait for phase `parity` of the barrier; false after `limit` cycles, or at once when
// `abort` is set (null: no abort check).
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, long long limit, const volatile int *abort) {
    const long long t0 = clock64();
    while (!bar_ready(bar, parity)) {
        if ((abort && *abort) || clock64() - t0 > limit) return false;
    }
    return true;
}

template <typename R, int NW>
__global__ void __launch_bounds__((NW + 1) * 32, kStreamCtasPerSm) pair_stream_kernel(
    int nclus, const int *__restrict__ cl0, const long long *__restrict__ cbase,
    const long long *__restrict__ cstart, long long total_vals, const long long *__restrict__ head,
    const int *__restrict__ count, const int *__restrict__ pair_j, const unsigned *__restrict__ masks,
    const long long *__restrict__ voff, const R *__restrict__ vals, const R *__restrict__ qc,
    R *__restrict__ ysum, long long limit, int withhold, int *__restrict__ err) {
    constexpr int S = kStreamStages, U = 16;
    constexpr long long E = sizeof(R);
    extern __shared__ __align__(128) unsigned char ring[];  // S stages of kStreamChunk bytes
    __shared__ __align__(8) uint64_t full[S], empty[S];
    __shared__ long long cst[S];  // absolute first byte of the chunk held by each stage
    __shared__ int abort_word;
    volatile int *abort_flag = &abort_word;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int I0 = cl0[blockIdx.x], I1 = cl0[blockIdx.x + 1];
    if (I0 >= I1) return;  // no clusters: the whole CTA leaves before any barrier
    const long long nch = cbase[blockIdx.x + 1] - cbase[blockIdx.x];
    const long long *cs = cstart + cbase[blockIdx.x];
    const long long B0 = voff[head[I0]] * E;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&empty[s])), "r"(NW) : "memory");
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (w == NW) {  // producer warp: lane 0 issues, the warp fetches chunk bounds 32 at a time
        if (withhold) return;  // a test of the bounded waits: nothing is issued, nothing arrives
        const long long B1 = (I1 < nclus ? voff[head[I1]] : total_vals) * E;
        long long issued = 0;
        bool ok = true;
        for (long long base = 0; base < nch && ok; base += 32) {
            const long long cl = base + lane;
            const long long lo_l = cl < nch ? cs[cl] : 0;
            const long long hi_l = cl + 1 < nch ? cs[cl + 1] : B1;
            const int nb = (int)min(32LL, nch - base);
            for (int l = 0; l < nb && ok; ++l) {
                const long long c = base + l;
                const long long lo = __shfl_sync(0xffffffffu, lo_l, l);
                const long long hi = __shfl_sync(0xffffffffu, hi_l, l);
                const int s = (int)(c % S);
                if (lane == 0) {
                    if (c >= S)
                        ok = bar_wait(smem_addr(&empty[s]), (uint32_t)((c / S - 1) & 1), limit, abort_flag);
                    if (ok) {
                        cst[s] = lo;
                        const uint32_t bytes = (uint32_t)(hi - lo);
                        const uint32_t fb = smem_addr(&full[s]);
                        if (bytes > 0) {
                            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(bytes)
                                         : "memory");
                            asm volatile(
                                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                                "[%3];" ::"r"(smem_addr(ring + (size_t)s * kStreamChunk)),
                                "l"(reinterpret_cast<const unsigned char *>(vals) + lo), "r"(bytes), "r"(fb)
                                : "memory");
                        } else {
                            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(fb) : "memory");
                        }
                        ++issued;
                    } else if (!*abort_flag) {
                        *abort_flag = 1;
                        atomicExch(err, 1);
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
            }
        }
        if (lane == 0)  // the copies of the last stages may still be in flight
            for (long long c = issued > S ? issued - S : 0; c < issued; ++c)
                bar_wait(smem_addr(&full[c % S]), (uint32_t)((c / S) & 1), kDrainLimit, nullptr);
        return;
    }

    // consumer warps: each waits for every chunk in order and releases every chunk below
    // the one holding its current pair as soon as it has waited for it (a warp never holds
    // a chunk while it waits for a later one, so the warp with the oldest chunk can always
    // go on)
    long long waited = 0, released = 0;  // chunks waited for / released by this warp
    bool ok = true;                      // warp-uniform
    auto release_below = [&](long long c) {
        __syncwarp();
        while (released < c && released < waited) {
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&empty[released % S]))
                             : "memory");
            ++released;
        }
    };
    // wait for the chunks up to c, releasing each one below `keep` once waited for
    auto advance = [&](long long c, long long keep) {
        while (ok && waited <= c) {
            const int s = (int)(waited % S);
            bool r = bar_wait(smem_addr(&full[s]), (uint32_t)((waited / S) & 1), limit, abort_flag);
            r = __all_sync(0xffffffffu, r);
            if (!r) {
                ok = false;
                if (lane == 0 && !*abort_flag) {
                    *abort_flag = 1;
                    atomicExch(err, 1);
                }
                break;
            }
            ++waited;
            release_below(min(keep, waited));
        }
        release_below(min(keep, waited));
    };

    long long h0 = head[I0];
    int n = count[I0];
    int Jc = 0;
    unsigned mc = 0;
    long long oc = 0;
    R xc = 0;
    if (w < n) {
        Jc = pair_j[h0 + w];
        mc = masks[(h0 + w) * CS + lane];
        oc = voff[h0 + w];
        xc = qc[Jc * CS + lane];
    }
    for (int I = I0; I < I1; ++I) {
        const long long h0n = I + 1 < I1 ? head[I + 1] : 0;
        const int nn = I + 1 < I1 ? count[I + 1] : 0;
        R yI = 0, yI2 = 0;  // FP32: odd slots into a second sum (half the dependent-add chain)
        for (int k = w; k < n; k += NW) {
            // the next pair of this warp (in this cluster or the next) while this one is summed
            long long pn = -1;
            if (k + NW < n)
                pn = h0 + k + NW;
            else if (w < nn)
                pn = h0n + w;
            int Jn = 0;
            unsigned mn = 0;
            long long on = 0;
            R xn = 0;
            if (pn >= 0) {
                Jn = pair_j[pn];
                mn = masks[pn * CS + lane];
                on = voff[pn];
                xn = qc[Jn * CS + lane];
            }
            if (ok) {
                const long long vb = oc * E;
                const long long c = min((vb - B0) >> kStreamShift, nch - 1);
                advance(c, c);
                if (ok) {
                    const int s = (int)(c % S);
                    unsigned m = mc;
                    const RowGroup g = row_group(m, lane);
                    const int rcur = RG == CS ? g.rows : (int)__reduce_max_sync(0xffffffffu, (unsigned)g.rows);
                    const R *v = reinterpret_cast<const R *>(ring + (size_t)s * kStreamChunk + (vb - cst[s])) + g.off;
                    for (int base = 0; base < rcur; base += U) {
                        R t[U];
#pragma unroll
                        for (int u = 0; u < U; ++u) t[u] = base + u < g.rows ? v[(base + u) * RG] : (R)0;
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            const int j = top_bit(m);
                            m = below_bit(m, j);
                            const R xj = __shfl_sync(0xffffffffu, xc, j);
                            if (sizeof(R) == 4 && (u & 1)) {
                                yI2 += t[u] * xj;
                            } else {
                                yI += t[u] * xj;
                            }
                        }
                    }
                }
            }
            Jc = Jn;
            mc = mn;
            oc = on;
            xc = xn;
        }
        if (w < n) atomicAdd(&ysum[(size_t)I * CS + lane], yI + yI2);  // this warp's part of cluster I
        if (w >= n && w < nn) {  // no pair of this warp in cluster I: fetch its first of the next
            Jc = pair_j[h0n + w];
            mc = masks[(h0n + w) * CS + lane];
            oc = voff[h0n + w];
            xc = qc[Jc * CS + lane];
        }
        h0 = h0n;
        n = nn;
    }
    // every chunk is waited for and released, so that the producer never waits in vain
    advance(nch - 1, nch);
}

// out_i = Phi_body(i) - (phik_i + self q_i + y_i) (or the bare sum when phi_body is NULL)
// from the streamed product's sums y in cluster order, which are cleared for the next one.
template <typename R>
__global__ void stream_finish_kernel(int nslots, const int *__restrict__ members, R *__restrict__ ysum,
                                     const R *__restrict__ q, const R *__restrict__ phik, double selfc,
                                     const double *__restrict__ phi_body, const uint32_t *__restrict__ body,
                                     double *__restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nslots) return;
    const int bi = members[k];
    const R y = ysum[k];
    ysum[k] = (R)0;
    if (bi < 0) return;
    write_row(out, bi, (double)y, phik, q, selfc, phi_body, body);
}

// CTA b of G takes the clusters whose first stored value lies in [T b/G, T (b+1)/G) of the
// T stored values (cluster boundaries), and one chunk per 8 KB window of its bytes (at
// least one).  One block of G <= 1024 threads.
__global__ void __launch_bounds__(1024) stream_split_kernel(int nclus, int G, const long long *__restrict__ head,
                                    const long long *__restrict__ voff, long long total_vals, int elem,
                                    int *__restrict__ cl0, long long *__restrict__ cbase) {
    typedef cub::BlockScan<long long, 1024> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int sc[1025];
    const int b = threadIdx.x;
    if (b < G) {
        const long long target = total_vals * b / G;
        int lo = 0, hi = nclus;  // first cluster whose first value is at or after target
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (voff[head[mid]] >= target)
                hi = mid;
            else
                lo = mid + 1;
        }
        sc[b] = b == 0 ? 0 : lo;
    }
    if (b == 0) sc[G] = nclus;
    __syncthreads();
    long long nchunks = 0;
    if (b < G) {
        const int a = sc[b], e = sc[b + 1];
        if (a < e) {
            const long long v0 = voff[head[a]];
            const long long v1 = e < nclus ? voff[head[e]] : total_vals;
            const long long bytes = (v1 - v0) * elem;
            nchunks = bytes > 0 ? ((bytes - 1) >> kStreamShift) + 1 : 1;
        }
        cl0[b] = sc[b];
    }
    if (b == 0) cl0[G] = nclus;
    long long off = 0, tot = 0;
    Scan(tmp).ExclusiveSum(nchunks, off, tot);
    if (b < G) cbase[b] = off;
    if (b == 0) cbase[G] = tot;
}

// First byte of every chunk: the first pair whose values start in the chunk's window
// (a window without a start gets the next start, i.e. an empty chunk; windows after the
// range's last start end at the range's end).
__global__ void stream_chunks_kernel(long long npairs, int G, int nclus, const int *__restrict__ pair_i,
                                     const int *__restrict__ cl0, const long long *__restrict__ cbase,
                                     const long long *__restrict__ head, const long long *__restrict__ voff,
                                     long long total_vals, int elem, long long *__restrict__ cstart) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int I = pair_i[p];
    int lo = 0, hi = G - 1;  // the last CTA whose first cluster is at or before I
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cl0[mid] <= I)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int b = lo;
    const long long first = head[cl0[b]];
    const long long last = (cl0[b + 1] < nclus ? head[cl0[b + 1]] : npairs) - 1;
    const long long B0 = voff[first] * elem;
    const long long nch = cbase[b + 1] - cbase[b];
    const long long k = min((voff[p] * elem - B0) >> kStreamShift, nch - 1);
    const long long kp = p == first ? -1 : min((voff[p - 1] * elem - B0) >> kStreamShift, nch - 1);
    for (long long kk = kp + 1; kk <= k; ++kk) cstart[cbase[b] + kk] = voff[p] * elem;
    if (p == last) {
        const long long B1 = (cl0[b + 1] < nclus ? voff[head[cl0[b + 1]]] : total_vals) * elem;
        for (long long kk = k + 1; kk < nch; ++kk) cstart[cbase[b] + kk] = B1;
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
            write_row(out, bi, (double)tot, phik, q, selfc, phi_body, body);
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
            const int j = top_bit(mm) & 31;
            mm = below_bit(mm, j);
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
        write_row(out, bi, tot, phik, q, selfc, phi_body, body);
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

template <typename R> R *ysum_of(RealSpace &r);
template <> float *ysum_of<float>(RealSpace &r) { return r.ysum32; }
template <> double *ysum_of<double>(RealSpace &r) { return r.ysum64; }
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

template <typename R> RealSpace::StreamPlan &plan_of(RealSpace &r);
template <> RealSpace::StreamPlan &plan_of<float>(RealSpace &r) { return r.plan32; }
template <> RealSpace::StreamPlan &plan_of<double>(RealSpace &r) { return r.plan64; }

bool streamed(const cr_handle *h) { return (h->rs_onfly & CR_REALSPACE_STREAM) != 0; }
// Cluster ranges and chunk starts of the streamed product of precision R (once per
// geometry, after the values): kStreamCtasPerSm CTAs per multiprocessor, at most one per
// cluster and at most 1024.
template <typename R> int stream_plan(cr_handle *h) {
    RealSpace &r = h->rs;
    RealSpace::StreamPlan &P = plan_of<R>(r);
    const int G = std::max(1, std::min(std::min(kStreamCtasPerSm * h->n_sm, r.nclus), 1024));
    if (!P.cl0) {
        CR_TRY(dalloc(h, &P.cl0, 1025));
        CR_TRY(dalloc(h, &P.cbase, 1025));
    }
    const long long need = ((r.nnz * (long long)sizeof(R)) >> kStreamShift) + G + 1;
    if (need > P.cap) {
        const long long cap = need + need / 8;
        CR_TRY(dalloc(h, &P.cstart, (size_t)cap));
        P.cap = cap;
    }
    // the ring's shared memory (64 KB) is above the default limit; set once per precision,
    // here, outside any stream capture
    static const cudaError_t attr = cudaFuncSetAttribute(
        pair_stream_kernel<R, kStreamWarps>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStreamStages * kStreamChunk);
    CR_CUDA(h, attr);
    stream_split_kernel<<<1, 1024, 0, h->stream>>>(r.nclus, G, r.head, r.voff, r.nnz, (int)sizeof(R), P.cl0, P.cbase);
    CR_LAUNCH(h, "stream_split_kernel");
    stream_chunks_kernel<<<blocks_for(r.npairs, 256), 256, 0, h->stream>>>(
        r.npairs, G, r.nclus, r.pair_i, P.cl0, P.cbase, r.head, r.voff, r.nnz, (int)sizeof(R), P.cstart);
    CR_LAUNCH(h, "stream_chunks_kernel");
    P.ctas = G;
    P.valid = true;
    return CR_OK;
}

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
    if (h->N == 0 || onfly<R>(h)) return CR_OK;
    if (valid_of<R>(r)) return streamed(h) && !plan_of<R>(r).valid ? stream_plan<R>(h) : CR_OK;
    if (h->user.precision != CR_FP64 && !r.valid32 && !r.valid64 && !onfly<float>(h) && !onfly<double>(h)) {
        CR_TRY(realspace_reserve<float>(h));
        CR_TRY(realspace_reserve<double>(h));
        pair_values_kernel<float, double><<<blocks_for(r.npairs * 32, 256), 256, 0, h->stream>>>(
            r.npairs, r.pair_i, r.pair_j, r.members, h->m64.pos, h->m64.phiq, rs_build(h), r.masks, r.voff,
            r.vals32, r.vals64);
        CR_LAUNCH(h, "pair_values_kernel");
        r.valid32 = r.valid64 = true;
        if (streamed(h)) {
            CR_TRY(stream_plan<float>(h));
            CR_TRY(stream_plan<double>(h));
        }
        return CR_OK;
    }
    CR_TRY(realspace_reserve<R>(h));
    pair_values_kernel<R><<<blocks_for(r.npairs * 32, 256), 256, 0, h->stream>>>(
        r.npairs, r.pair_i, r.pair_j, r.members, h->m64.pos, h->m64.phiq, rs_build(h), r.masks, r.voff,
        blocks_of<R>(r));
    CR_LAUNCH(h, "pair_values_kernel");
    valid_of<R>(r) = true;
    if (streamed(h)) CR_TRY(stream_plan<R>(h));
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
    dfree(&r.ysum32);
    dfree(&r.ysum64);
    dfree(&r.freal);
    dfree(&r.bits);
    dfree(&r.boff);
    dfree(&r.pshift);
    dfree(&r.err);
    for (RealSpace::StreamPlan *P : {&r.plan32, &r.plan64}) {
        dfree(&P->cl0);
        dfree(&P->cbase);
        dfree(&P->cstart);
        *P = RealSpace::StreamPlan{};
    }
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
    CR_TRY(dalloc(h, &r.ysum32, nc * CS));
    CR_TRY(dalloc(h, &r.ysum64, nc * CS));
    CR_CUDA(h, cudaMemsetAsync(r.ysum32, 0, nc * CS * sizeof(float), h->stream));
    CR_CUDA(h, cudaMemsetAsync(r.ysum64, 0, nc * CS * sizeof(double), h->stream));
    CR_TRY(dalloc(h, &r.freal, 3 * (size_t)std::max(h->N, 1)));
    CR_TRY(dalloc(h, &r.bits, 1));
    CR_TRY(dalloc(h, &r.boff, nc * CS));
    CR_TRY(dalloc(h, &r.err, 1));
    CR_CUDA(h, cudaMemsetAsync(r.err, 0, sizeof(int), h->stream));
    if (!h->side) {  // the wave-space branch of the operator: highest stream priority
        int least = 0, greatest = 0;
        CR_CUDA(h, cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CR_CUDA(h, cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, greatest));
        CR_CUDA(h, cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
        CR_CUDA(h, cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    }
    return CR_OK;
}

// Clusters and cluster pairs of the current positions; blocks are filled on first
// use per precision.
int realspace_build(cr_handle *h) {
    RealSpace &r = h->rs;
    const int N = h->N;
    r.valid32 = r.valid64 = false;
    r.plan32.valid = r.plan64.valid = false;
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
                                            r.extent, r.boff, r.pshift);
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

template <typename R>
int real_space_apply(cr_handle *h, MeshBuffers<R> &m, const double *phi_body, double *out, bool rows_only) {
    const int N = h->N;
    if (N == 0) return CR_OK;
    RealSpace &r = h->rs;
    {
        ProfScope pb(h, PROF_GEOMETRY);
        CR_TRY(realspace_blocks<R>(h));
    }
    ProfScope ps(h, PROF_REAL);
    const R *phik = rows_only ? nullptr : m.phi;  // NULL: the real-space sums only
    R *qc = acc_of<R>(r);
    gather_cluster_kernel<R><<<blocks_for((long)r.nclus * CS, 256), 256, 0, h->stream>>>(r.nclus * CS, r.members,
                                                                                         m.q, qc);
    CR_LAUNCH(h, "gather_cluster_kernel");
    constexpr int W = kSpmvWarps;
    if (onfly<R>(h)) {
        if constexpr (sizeof(R) == 4) {
            pair_otf32_kernel<W><<<r.nclus, W * 32, onfly32_smem(h), h->stream>>>(
                r.head, r.count, r.pair_j, r.members, r.masks, r.boff, r.pshift, rs_build(h), h->m32.phiq,
                (float)(h->d.n_table / (h->d.rcut - h->d.dr)), qc, m.q, phik, h->d.selfcoeff, phi_body, h->d_body,
                out);
            CR_LAUNCH(h, "pair_otf32_kernel");
        } else {
            pair_otf64_kernel<W><<<r.nclus, W * 32, 0, h->stream>>>(r.head, r.count, r.pair_j, r.members, r.masks,
                                                                    h->m64.pos, h->m64.phiq, rs_build(h), qc, m.q,
                                                                    phik, h->d.selfcoeff, phi_body, h->d_body, out);
            CR_LAUNCH(h, "pair_otf64_kernel");
        }
        return CR_OK;
    }
    if (streamed(h)) {
        const RealSpace::StreamPlan &P = plan_of<R>(r);
        constexpr int NW = kStreamWarps;
        const size_t smem = (size_t)kStreamStages * kStreamChunk;
        R *ysum = ysum_of<R>(r);
        pair_stream_kernel<R, NW><<<P.ctas, (NW + 1) * 32, smem, h->stream>>>(
            r.nclus, P.cl0, P.cbase, P.cstart, r.nnz, r.head, r.count, r.pair_j, r.masks, r.voff, blocks_of<R>(r),
            qc, ysum, r.wait_limit, r.withhold_next, r.err);
        r.withhold_next = 0;
        CR_LAUNCH(h, "pair_stream_kernel");
        stream_finish_kernel<R><<<blocks_for((long)r.nclus * CS, 256), 256, 0, h->stream>>>(
            r.nclus * CS, r.members, ysum, m.q, phik, h->d.selfcoeff, phi_body, h->d_body, out);
        CR_LAUNCH(h, "stream_finish_kernel");
        return CR_OK;
    }
    pair_spmv_kernel<R, W, 16><<<r.nclus, W * 32, 0, h->stream>>>(
        r.nclus, r.head, r.count, r.pair_j, r.members, r.masks, r.voff, r.nnz_pair, blocks_of<R>(r), qc, m.q, phik,
        h->d.selfcoeff, phi_body, h->d_body, out);
    CR_LAUNCH(h, "pair_spmv_kernel");
    return CR_OK;
}

// Adds the wave-space part and the self term to rows that hold only their real-space sums
// (real_space_apply with rows_only).
template <typename R> int real_space_rows(cr_handle *h, MeshBuffers<R> &m, const double *phi_body, double *out) {
    if (h->N == 0) return CR_OK;
    rows_combine_kernel<R><<<blocks_for(h->N, 256), 256, 0, h->stream>>>(h->N, m.phi, m.q, h->d.selfcoeff, phi_body,
                                                                        h->d_body, out);
    CR_LAUNCH(h, "rows_combine_kernel");
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

int realspace_check(cr_handle *h) {
    RealSpace &r = h->rs;
    if (!r.err) return CR_OK;
    int e = 0;
    CR_CUDA(h, cudaMemcpyAsync(&e, r.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    if (e == 0) return CR_OK;
    CR_CUDA(h, cudaMemsetAsync(r.err, 0, sizeof(int), h->stream));
    return fail(h, CR_TIMEOUT, "real-space product: a bounded device wait ran out");
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

// ---- lockstep batches ----------------------------------------------------------------
// The real-space stages of a batched operator application: charges in cluster order, the
// stored-value product (the same per-cluster body as pair_spmv_kernel) writing the bare
// sums into the rows of the output vector, then the rows combined with the wave-space
// part and the self term.

namespace {

template <typename R>
__global__ void gather_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                    const int *__restrict__ mask) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &b = reps[it.x];
    const int k = it.y * blockDim.x + threadIdx.x;
    if (k >= b.nclus * CS) return;
    const int i = b.members[k];
    brep_acc<R>(b)[k] = i >= 0 ? brep_q<R>(b)[i] : (R)0;
}

template <typename R, int W, int U>
__global__ void __launch_bounds__(W * 32, sizeof(R) == 4 ? 6 : 1)
    spmv_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items, const int *__restrict__ mask,
                      int yout) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &b = reps[it.x];
    pair_spmv_cluster<R, W, U>(it.y, b.head, b.count, b.pair_j, b.members, b.masks, b.voff, b.slots, brep_vals<R>(b),
                               brep_acc<R>(b), brep_q<R>(b), nullptr, b.selfc, nullptr, b.body, b.vec[yout]);
}

template <typename R>
__global__ void rows_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                  const int *__restrict__ mask, int xin, int yout) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &b = reps[it.x];
    double *out = b.vec[yout];
    const double *phi_body = b.vec[xin] + b.N;
    const R *phik = brep_phi<R>(b), *q = brep_q<R>(b);
    for (int i = it.y * blockDim.x + threadIdx.x; i < b.N; i += b.vblk * blockDim.x)
        write_row(out, i, out[i], phik, q, b.selfc, phi_body, b.body);
}

}  // namespace

template <typename R> int batch_real(cr_batch *bt, const int *mask, int yout, cudaStream_t s) {
    if (bt->n_items[BL_CLELEMS] > 0) {
        gather_batch_kernel<R><<<bt->n_items[BL_CLELEMS], 256, 0, s>>>(bt->d_reps, bt->d_items[BL_CLELEMS], mask);
        ++bt->launches;
        CR_TRY(batch_check(bt, cudaGetLastError(), "gather_batch_kernel"));
    }
    if (bt->n_items[BL_CLUSTERS] > 0) {
        constexpr int W = kSpmvWarps;
        spmv_batch_kernel<R, W, 16><<<bt->n_items[BL_CLUSTERS], W * 32, 0, s>>>(bt->d_reps, bt->d_items[BL_CLUSTERS],
                                                                                mask, yout);
        ++bt->launches;
        CR_TRY(batch_check(bt, cudaGetLastError(), "spmv_batch_kernel"));
    }
    return CR_OK;
}

template <typename R> int batch_rows(cr_batch *bt, const int *mask, int xin, int yout, cudaStream_t s) {
    if (bt->n_items[BL_VEC] == 0) return CR_OK;
    rows_batch_kernel<R><<<bt->n_items[BL_VEC], 256, 0, s>>>(bt->d_reps, bt->d_items[BL_VEC], mask, xin, yout);
    ++bt->launches;
    return batch_check(bt, cudaGetLastError(), "rows_batch_kernel");
}

template int batch_real<float>(cr_batch *, const int *, int, cudaStream_t);
template int batch_real<double>(cr_batch *, const int *, int, cudaStream_t);
template int batch_rows<float>(cr_batch *, const int *, int, int, cudaStream_t);
template int batch_rows<double>(cr_batch *, const int *, int, int, cudaStream_t);

template int real_space_apply<float>(cr_handle *, MeshBuffers<float> &, const double *, double *, bool);
template int real_space_apply<double>(cr_handle *, MeshBuffers<double> &, const double *, double *, bool);
template int real_space_rows<float>(cr_handle *, MeshBuffers<float> &, const double *, double *);
template int real_space_rows<double>(cr_handle *, MeshBuffers<double> &, const double *, double *);
template int real_space_force<float>(cr_handle *, MeshBuffers<float> &, const double *, double *);
template int real_space_force<double>(cr_handle *, MeshBuffers<double> &, const double *, double *);

}  // namespace cr
