// mesh.cu -- wave-space part of the operator: spread, FFT, influence function,
// inverse FFT, contract (ConductorRigid.cu:144-466, 919-937, 1256-1274).
//
// Layout: real mesh [Nx][Ny][Nz] (x slowest, the reference's i*Ny*Nz + j*Nz + k,
// ConductorRigid.cu:229), half spectrum [Nx][Ny][Nz/2+1] from an R2C/D2Z transform.
// The reference transforms the real charge mesh with a full C2C FFT and keeps the
// real part of the inverse; with a real, even influence function the half-spectrum
// pair R2C/C2R gives the same numbers with half the traffic.
//
// Spread and contract work on tiles of T^3 mesh nodes.  Beads are binned by the tile
// that holds the first node of their P^3 window; one CTA owns a tile and a
// (T+P-1)^3 shared-memory halo buffer.  Spread accumulates every bead of the tile in
// the buffer with shared-memory atomics and adds the buffer to the mesh once; contract
// loads the buffer once and serves all beads of the tile from shared memory.  One
// warp handles one bead: lanes compute the 3P separable Gaussian factors
// exp(-2 xi^2 r_d^2 / eta_d) (the reference evaluates exp of their sum per node,
// ConductorRigid.cu:219-223), then sweep the P^2 (y,z) columns with the x loop inside.
#include <cub/cub.cuh>

#include <type_traits>

#include <algorithm>
#include <mutex>

#include "cr_internal.cuh"

namespace cr {

namespace {

template <typename R> struct Vec3 { R x, y, z; };

struct MeshShape {
    int Ng[3];     // mesh nodes per dimension
    int ntd[3];    // tiles per dimension
    int T;         // tile edge
    int P;         // support
    int Bd;        // halo buffer edge T + P - 1
    int zp;        // z pitch of the contraction halo buffer
};

// z pitch of the contraction halo buffer: P + 32 (>= T + P - 1 for T <= 32, and congruent
// to P modulo 32, so that the P*P window columns a warp reads in order fall on distinct
// banks) where that buffer fits in 227 KB of shared memory, else T + P - 1.
inline int contract_pitch(int T, int P, size_t elem) {
    const size_t Bd = (size_t)T + P - 1;
    const size_t padded = (Bd * Bd * (P + 32) + 8 * 6 * (size_t)P) * elem;
    return padded <= 227 * 1024 ? P + 32 : (int)Bd;
}

template <typename R> struct WindowConst {
    R h[3], halfL[3], inv_eta[3];
    R xiterm;
};

__device__ __forceinline__ int wrapmod(int s, int n) {
    int r = s % n;
    return r < 0 ? r + n : r;
}

__device__ __forceinline__ float dexp(float x) { return __expf(x); }
__device__ __forceinline__ double dexp(double x) { return exp(x); }

template <typename R> __device__ __forceinline__ R warp_sum(R v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per-warp Gaussian factors for one bead: w[d*P + t] = exp(-xiterm (node - x)^2 / eta_d)
// with node = h_d (start_d + t) - L_d/2 (ConductorRigid.cu:212-223); u[d*P + t] =
// (x - node)/eta_d for the force.
template <typename R, bool WANT_U>
__device__ __forceinline__ void window_factors(const WindowConst<R> &wc, int P, R px, R py, R pz, int4 s,
                                               R *w, R *u, int lane) {
    for (int t = lane; t < 3 * P; t += 32) {
        int d = t >= 2 * P ? 2 : (t >= P ? 1 : 0);
        int tt = t - d * P;
        R x = d == 0 ? px : (d == 1 ? py : pz);
        int st = d == 0 ? s.x : (d == 1 ? s.y : s.z);
        R r = wc.h[d] * (R)(st + tt) - wc.halfL[d] - x;
        w[t] = dexp(-wc.xiterm * r * r * wc.inv_eta[d]);
        if (WANT_U) u[t] = -r * wc.inv_eta[d];
    }
}

// Index of mesh node g (tile origin + buffer offset, g >= 0) folded into [0, n).
__device__ __forceinline__ int fold(int g, int n) {
    while (g >= n) g -= n;
    return g;
}

// PT > 0: support and tile fixed at compile time (T = 8); PT == 0: runtime values.
template <typename R, int PT>
__global__ void __launch_bounds__(256) spread_tiles_kernel(
    const typename Prec<R>::R4 *__restrict__ pos, const R *__restrict__ q, const int4 *__restrict__ wstart,
    const int *__restrict__ tile_start, const int *__restrict__ tile_beads, MeshShape ms, WindowConst<R> wc,
    R prefac, R *__restrict__ grid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *buf = reinterpret_cast<R *>(smem_raw);
    const int P = PT ? PT : ms.P;
    const int T = PT ? 8 : ms.T;
    const int Bd = PT ? 8 + PT - 1 : ms.Bd;
    const int nbuf = Bd * Bd * Bd;
    const int tile = blockIdx.x;
    const int b0 = tile_start[tile], b1 = tile_start[tile + 1];
    if (b0 == b1) return;  // uniform across the block
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    R *w = buf + nbuf + warp * 3 * P;
    for (int i = threadIdx.x; i < nbuf; i += blockDim.x) buf[i] = (R)0;
    __syncthreads();
    const int tz = tile % ms.ntd[2], ty = (tile / ms.ntd[2]) % ms.ntd[1], tx = tile / (ms.ntd[2] * ms.ntd[1]);
    for (int k = b0 + warp; k < b1; k += nw) {
        const int i = tile_beads[k];
        const typename Prec<R>::R4 p = pos[i];
        const int4 s = wstart[i];
        window_factors<R, false>(wc, P, p.x, p.y, p.z, s, w, nullptr, lane);
        __syncwarp();
        const int ox = wrapmod(s.x, ms.Ng[0]) - tx * T;
        const int oy = wrapmod(s.y, ms.Ng[1]) - ty * T;
        const int oz = wrapmod(s.z, ms.Ng[2]) - tz * T;
        const R c = prefac * q[i];
        if (ox >= 0 && ox < T && oy >= 0 && oy < T && oz >= 0 && oz < T) {
            for (int e = lane; e < P * P; e += 32) {
                const int b = e / P, cc = e - b * P;
                const R wyz = c * w[P + b] * w[2 * P + cc];
                R *col = buf + ((size_t)ox * Bd + (oy + b)) * Bd + (oz + cc);
                for (int a = 0; a < P; ++a) atomicAdd(col + (size_t)a * Bd * Bd, wyz * w[a]);
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int n = threadIdx.x; n < nbuf; n += blockDim.x) {
        const R v = buf[n];
        if (v == (R)0) continue;
        const int bz = n % Bd, by = (n / Bd) % Bd, bx = n / (Bd * Bd);
        const int gx = fold(tx * T + bx, ms.Ng[0]);
        const int gy = fold(ty * T + by, ms.Ng[1]);
        const int gz = fold(tz * T + bz, ms.Ng[2]);
        atomicAdd(grid + ((size_t)gx * ms.Ng[1] + gy) * ms.Ng[2] + gz, v);
    }
}

// Spread for a compile-time support PT (tile edge 8, halo buffer edge BD = 8 + PT - 1):
// thread t < BD*BD owns the buffer column (y, z) = (t / BD, t % BD) in registers.  Beads
// of the tile are taken 32 at a time: the first threads stage the batch's bead data, then
// all threads compute the batch's 32 x 3P Gaussian factors into shared memory (x factors
// already shifted to the column's x index and scaled by prefac q), then every thread adds
// the beads whose window covers its column.  No shared-memory atomics; within a tile the
// summation order is fixed.  The columns are added to the mesh once at the end.
// (one tile: the body of spread_columns_kernel and of its lockstep-batch form)
template <typename R, int PT>
__device__ __forceinline__ void spread_columns_tile(
    int tile, const typename Prec<R>::R4 *__restrict__ pos, const R *__restrict__ q, const int4 *__restrict__ wstart,
    const int *__restrict__ tile_start, const int *__restrict__ tile_beads, MeshShape ms, WindowConst<R> wc,
    R prefac, R *__restrict__ grid) {
    constexpr int P = PT, T = 8, BD = T + PT - 1;
    __shared__ R sx[32][BD];     // shifted, scaled x factors
    __shared__ R sy[32][P], sz[32][P];
    __shared__ R sp[32][3], sc[32];
    __shared__ int4 sst[32];
    __shared__ int sox[32], soy[32], soz[32];
    const int b0 = tile_start[tile], b1 = tile_start[tile + 1];
    if (b0 == b1) return;
    const int t = threadIdx.x;
    const int cy = t / BD, cz = t - (t / BD) * BD;
    const bool owner = t < BD * BD;
    const int tz = tile % ms.ntd[2], ty = (tile / ms.ntd[2]) % ms.ntd[1], tx = tile / (ms.ntd[2] * ms.ntd[1]);
    R col[BD];
#pragma unroll
    for (int x = 0; x < BD; ++x) col[x] = (R)0;
    for (int base = b0; base < b1; base += 32) {
        const int nb = min(32, b1 - base);
        // bead data of the batch, and cleared x-factor rows
        if (t < nb) {
            const int i = tile_beads[base + t];
            const typename Prec<R>::R4 p = pos[i];
            const int4 st = wstart[i];
            const int ox = wrapmod(st.x, ms.Ng[0]) - tx * T;
            const int oy = wrapmod(st.y, ms.Ng[1]) - ty * T;
            const int oz = wrapmod(st.z, ms.Ng[2]) - tz * T;
            const bool ok = ox >= 0 && ox < T && oy >= 0 && oy < T && oz >= 0 && oz < T;
            sp[t][0] = p.x;
            sp[t][1] = p.y;
            sp[t][2] = p.z;
            sst[t] = st;
            sc[t] = ok ? prefac * q[i] : (R)0;
            sox[t] = ok ? ox : -1;   // a bead outside its tile writes no x factor...
            soy[t] = ok ? oy : -BD;  // ...and touches no column
            soz[t] = oz;
        }
        for (int e = t; e < nb * BD; e += blockDim.x) (&sx[0][0])[e] = (R)0;
        __syncthreads();
        // the batch's Gaussian factors, all threads: entry e = (bead l, dimension d, node a)
        for (int e = t; e < nb * 3 * P; e += blockDim.x) {
            const int l = e / (3 * P), rem = e - l * 3 * P;
            const int d = rem / P, a = rem - d * P;
            // (selected, not indexed, so the parameter block stays in registers)
            const int st = d == 0 ? sst[l].x : (d == 1 ? sst[l].y : sst[l].z);
            const R hd = d == 0 ? wc.h[0] : (d == 1 ? wc.h[1] : wc.h[2]);
            const R half = d == 0 ? wc.halfL[0] : (d == 1 ? wc.halfL[1] : wc.halfL[2]);
            const R ie = d == 0 ? wc.inv_eta[0] : (d == 1 ? wc.inv_eta[1] : wc.inv_eta[2]);
            const R r = hd * (R)(st + a) - half - sp[l][d];
            const R w = dexp(-wc.xiterm * r * r * ie);
            if (d == 0) {
                if (sox[l] >= 0) sx[l][sox[l] + a] = sc[l] * w;
            } else if (d == 1) {
                sy[l][a] = w;
            } else {
                sz[l][a] = w;
            }
        }
        __syncthreads();
        if (owner) {
            for (int b = 0; b < nb; ++b) {
                const int ay = cy - soy[b], az = cz - soz[b];
                if ((unsigned)ay < (unsigned)P && (unsigned)az < (unsigned)P) {
                    const R wyz = sy[b][ay] * sz[b][az];
#pragma unroll
                    for (int x = 0; x < BD; ++x) col[x] += wyz * sx[b][x];
                }
            }
        }
        __syncthreads();
    }
    if (owner) {
        const int gy = fold(ty * T + cy, ms.Ng[1]);
        const int gz = fold(tz * T + cz, ms.Ng[2]);
#pragma unroll
        for (int x = 0; x < BD; ++x) {
            if (col[x] != (R)0) {
                const int gx = fold(tx * T + x, ms.Ng[0]);
                atomicAdd(grid + ((size_t)gx * ms.Ng[1] + gy) * ms.Ng[2] + gz, col[x]);
            }
        }
    }
}

template <typename R, int PT>
__global__ void __launch_bounds__(((8 + PT - 1) * (8 + PT - 1) + 31) / 32 * 32) spread_columns_kernel(
    const typename Prec<R>::R4 *__restrict__ pos, const R *__restrict__ q, const int4 *__restrict__ wstart,
    const int *__restrict__ tile_start, const int *__restrict__ tile_beads, MeshShape ms, WindowConst<R> wc,
    R prefac, R *__restrict__ grid) {
    spread_columns_tile<R, PT>(blockIdx.x, pos, q, wstart, tile_start, tile_beads, ms, wc, prefac, grid);
}

// (one tile: the body of contract_tiles_kernel and of its lockstep-batch form)
template <typename R, bool FORCE, int PT>
__device__ __forceinline__ void contract_tile(
    int tile, const typename Prec<R>::R4 *__restrict__ pos, const R *__restrict__ q, const int4 *__restrict__ wstart,
    const int *__restrict__ tile_start, const int *__restrict__ tile_beads, MeshShape ms, WindowConst<R> wc,
    R coeff, const R *__restrict__ grid, R *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *buf = reinterpret_cast<R *>(smem_raw);
    const int P = PT ? PT : ms.P;
    const int T = PT ? 8 : ms.T;
    const int Bd = PT ? 8 + PT - 1 : ms.Bd;
    // halo buffer [x][y][z] with the z rows at a pitch of P + 32 (>= Bd): column (b, c) of
    // a window then sits at bank (b * P + c) mod 32, so a warp reading P*P columns in
    // order touches 32 distinct banks
    const int zp = ms.zp;
    const int plane = Bd * zp;
    const int nbuf = Bd * plane;
    const int b0 = tile_start[tile], b1 = tile_start[tile + 1];
    if (b0 == b1) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    R *w = buf + nbuf + warp * 6 * P;
    R *u = w + 3 * P;
    const int tz = tile % ms.ntd[2], ty = (tile / ms.ntd[2]) % ms.ntd[1], tx = tile / (ms.ntd[2] * ms.ntd[1]);
    // fill: one (y, z) column per thread, x marched with an incremental fold
    for (int cidx = threadIdx.x; cidx < Bd * Bd; cidx += blockDim.x) {
        const int by = cidx / Bd, bz = cidx - by * Bd;
        const int gy = fold(ty * T + by, ms.Ng[1]);
        const int gz = fold(tz * T + bz, ms.Ng[2]);
        const R *src = grid + (size_t)gy * ms.Ng[2] + gz;
        const size_t xstride = (size_t)ms.Ng[1] * ms.Ng[2];
        int gx = fold(tx * T, ms.Ng[0]);
        R *dst = buf + by * zp + bz;
        for (int bx = 0; bx < Bd; ++bx) {
            dst[bx * plane] = src[(size_t)gx * xstride];
            if (++gx == ms.Ng[0]) gx = 0;
        }
    }
    __syncthreads();
    for (int k = b0 + warp; k < b1; k += nw) {
        const int i = tile_beads[k];
        const typename Prec<R>::R4 p = pos[i];
        const int4 s = wstart[i];
        window_factors<R, FORCE>(wc, P, p.x, p.y, p.z, s, w, u, lane);
        __syncwarp();
        const int ox = wrapmod(s.x, ms.Ng[0]) - tx * T;
        const int oy = wrapmod(s.y, ms.Ng[1]) - ty * T;
        const int oz = wrapmod(s.z, ms.Ng[2]) - tz * T;
        R acc = 0, fx = 0, fy = 0, fz = 0;
        if (ox >= 0 && ox < T && oy >= 0 && oy < T && oz >= 0 && oz < T) {
            for (int e = lane; e < P * P; e += 32) {
                const int b = e / P, cc = e - b * P;
                const R wyz = w[P + b] * w[2 * P + cc];
                const R *col = buf + (size_t)ox * plane + (oy + b) * zp + (oz + cc);
                R s0 = 0, sx = 0;
                for (int a = 0; a < P; ++a) {
                    const R g = w[a] * col[(size_t)a * plane];
                    s0 += g;
                    if (FORCE) sx += g * u[a];
                }
                if (FORCE) {
                    fx += wyz * sx;
                    fy += wyz * s0 * u[P + b];
                    fz += wyz * s0 * u[2 * P + cc];
                } else {
                    acc += wyz * s0;
                }
            }
        }
        if (FORCE) {
            fx = warp_sum(fx);
            fy = warp_sum(fy);
            fz = warp_sum(fz);
            if (lane == 0) {
                const R c = coeff * q[i];  // 2 quadW prefac xiterm q_i (ConductorRigid.cu:449,1274)
                out[3 * (size_t)i + 0] = c * fx;
                out[3 * (size_t)i + 1] = c * fy;
                out[3 * (size_t)i + 2] = c * fz;
            }
        } else {
            acc = warp_sum(acc);
            if (lane == 0) out[i] = coeff * acc;  // quadW prefac (ConductorRigid.cu:936-937)
        }
        __syncwarp();
    }
}

template <typename R, bool FORCE, int PT>
__global__ void __launch_bounds__(256) contract_tiles_kernel(
    const typename Prec<R>::R4 *__restrict__ pos, const R *__restrict__ q, const int4 *__restrict__ wstart,
    const int *__restrict__ tile_start, const int *__restrict__ tile_beads, MeshShape ms, WindowConst<R> wc,
    R coeff, const R *__restrict__ grid, R *__restrict__ out) {
    contract_tile<R, FORCE, PT>(blockIdx.x, pos, q, wstart, tile_start, tile_beads, ms, wc, coeff, grid, out);
}

template <typename R, typename C>
__global__ void scale_kernel(C *__restrict__ spec, const R *__restrict__ scale, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const R s = scale[i];
        C v = spec[i];
        v.x *= s;
        v.y *= s;
        spec[i] = v;
    }
}

// Influence function on the half spectrum (ConductorRigid.cc:245-274): for k != 0,
// j0(|k|)^2 exp(-sum_d (1 - eta_d) k_d^2 / (4 xi^2)) / |k|^2 / Ngrid with j0 = sin x / x.
template <typename R>
__global__ void scale_init_kernel(R *scale, int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                                  double ex, double ey, double ez, double xi) {
    const int Nzh = Nz / 2 + 1;
    const long n = (long)Nx * Ny * Nzh;
    long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const int k = (int)(idx % Nzh);
    const int j = (int)((idx / Nzh) % Ny);
    const int i = (int)(idx / ((long)Nzh * Ny));
    const double kx = ((i < (Nx + 1) / 2) ? i : i - Nx) * 2.0 * kPi / Lx;
    const double ky = ((j < (Ny + 1) / 2) ? j : j - Ny) * 2.0 * kPi / Ly;
    const double kz = ((k < (Nz + 1) / 2) ? k : k - Nz) * 2.0 * kPi / Lz;
    const double k2 = kx * kx + ky * ky + kz * kz;
    if (i == 0 && j == 0 && k == 0) {
        scale[idx] = (R)0;
        return;
    }
    const double etak2 = (1.0 - ex) * kx * kx + (1.0 - ey) * ky * ky + (1.0 - ez) * kz * kz;
    const double kk = sqrt(k2);
    const double j0 = sin(kk) / kk;
    scale[idx] = (R)(j0 * j0 * exp(-etak2 / (4.0 * xi * xi)) / k2 / ((double)Nx * Ny * Nz));
}

// Wave-space virial of U_k = 1/2 quadW sum_k S(k) |H(k)|^2 (H the spread mesh's
// transform, S the influence function, the sum over the full spectrum: modes of the half
// spectrum with 0 < kz < Nz/2 count twice).  Under the affine strain r -> (1 + e) r of
// positions and box, with the shell radius fixed, -dU_k/de_ab = sum_k E_k (delta_ab +
// g(k) k_a k_b / k^2), g = d ln S / d ln k = 2 k cot k - 4 - k^2 / (2 xi^2) for the
// continuous kernel j0(k)^2 exp(-k^2 / 4 xi^2) / k^2 (the Gaussian splitting factors of
// the spread and of S combine to it).  Per block: the six tensor components and E_k summed
// into partial[block][7] (the seventh the wave energy itself).
__global__ void wave_virial_kernel(const double2 *__restrict__ spec, const double *__restrict__ scale, int Nx,
                                   int Ny, int Nz, double Lx, double Ly, double Lz, double xi, double half_quadW,
                                   double *__restrict__ partial) {
    const int Nzh = Nz / 2 + 1;
    const long n = (long)Nx * Ny * Nzh;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        const int k = (int)(idx % Nzh);
        const int j = (int)((idx / Nzh) % Ny);
        const int i = (int)(idx / ((long)Nzh * Ny));
        if (i == 0 && j == 0 && k == 0) continue;
        const double kx = ((i < (Nx + 1) / 2) ? i : i - Nx) * 2.0 * kPi / Lx;
        const double ky = ((j < (Ny + 1) / 2) ? j : j - Ny) * 2.0 * kPi / Ly;
        const double kz = ((k < (Nz + 1) / 2) ? k : k - Nz) * 2.0 * kPi / Lz;
        const double k2 = kx * kx + ky * ky + kz * kz;
        const double2 hk = spec[idx];
        const double w = (k == 0 || (Nz % 2 == 0 && k == Nz / 2)) ? 1.0 : 2.0;
        const double E = half_quadW * w * scale[idx] * (hk.x * hk.x + hk.y * hk.y);
        const double kk = sqrt(k2);
        const double sk = sin(kk), ck = cos(kk);
        const double cot_term = fabs(sk) > 1e-300 ? 2.0 * kk * ck / sk : 0.0;  // E = 0 where sin k = 0
        const double g = (cot_term - 4.0 - k2 / (2.0 * xi * xi)) / k2;
        acc[0] += E * (1.0 + g * kx * kx);
        acc[1] += E * g * kx * ky;
        acc[2] += E * g * kx * kz;
        acc[3] += E * (1.0 + g * ky * ky);
        acc[4] += E * g * ky * kz;
        acc[5] += E * (1.0 + g * kz * kz);
        acc[6] += E;
    }
    __shared__ double red[8][7];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = 0; c < 7; ++c) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double t = 0.0;
        for (int v = 0; v < (int)(blockDim.x >> 5); ++v) t += red[v][threadIdx.x];
        partial[(size_t)blockIdx.x * 7 + threadIdx.x] = t;
    }
}

template <typename R> __global__ void cast_kernel(const double *__restrict__ in, R *__restrict__ out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (R)in[i];
}

template <typename R> MeshShape mesh_shape(const cr_handle *h) {
    MeshShape ms;
    for (int d = 0; d < 3; ++d) {
        ms.Ng[d] = h->d.grid[d];
        ms.ntd[d] = h->ntiles_dim[d];
    }
    ms.T = h->tile;
    ms.P = h->d.support;
    ms.Bd = h->tile + h->d.support - 1;
    ms.zp = contract_pitch(h->tile, h->d.support, sizeof(R));
    return ms;
}

template <typename R> WindowConst<R> window_const(const cr_handle *h) {
    WindowConst<R> wc;
    for (int d = 0; d < 3; ++d) {
        wc.h[d] = (R)h->d.h[d];
        wc.halfL[d] = (R)(0.5 * h->L[d]);
        wc.inv_eta[d] = (R)(1.0 / h->d.eta[d]);
    }
    wc.xiterm = (R)h->d.xiterm;
    return wc;
}

template <typename R> size_t spread_smem(const cr_handle *h) {
    const int Bd = h->tile + h->d.support - 1;
    return ((size_t)Bd * Bd * Bd + 8 * 3 * (size_t)h->d.support) * sizeof(R);
}
template <typename R> size_t contract_smem(const cr_handle *h) {
    const int Bd = h->tile + h->d.support - 1;
    return ((size_t)Bd * Bd * contract_pitch(h->tile, h->d.support, sizeof(R)) + 8 * 6 * (size_t)h->d.support) *
           sizeof(R);
}

// The dynamic shared-memory limit is a process-wide attribute of each kernel: it only
// ever grows (under a lock), so handles with different supports can launch concurrently.
std::mutex g_smem_mu;

template <typename R, int PT> int set_smem_attrs(cr_handle *h, size_t s1, size_t s2) {
    static size_t set1 = 0, set2 = 0;
    std::lock_guard<std::mutex> lk(g_smem_mu);
    if (s1 > set1) {
        CR_CUDA(h, cudaFuncSetAttribute(spread_tiles_kernel<R, PT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)s1));
        set1 = s1;
    }
    if (s2 > set2) {
        CR_CUDA(h, cudaFuncSetAttribute(contract_tiles_kernel<R, false, PT>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s2));
        CR_CUDA(h, cudaFuncSetAttribute(contract_tiles_kernel<R, true, PT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)s2));
        set2 = s2;
    }
    return CR_OK;
}

// Compile-time support for the common supports (tile edge 8), runtime otherwise.
template <typename R, typename F> int with_support(const cr_handle *h, F f) {
    if (h->tile == 8 && h->d.support == 9) return f(std::integral_constant<int, 9>());
    if (h->tile == 8 && h->d.support == 11) return f(std::integral_constant<int, 11>());
    return f(std::integral_constant<int, 0>());
}

}  // namespace

template <typename R> int mesh_init(cr_handle *h, MeshBuffers<R> &m) {
    typedef typename Prec<R>::R4 R4;
    typedef typename Prec<R>::R2 R2;
    typedef typename Prec<R>::C C;
    mesh_free(m);
    const int N = h->N;
    const long G = grid_size(h), S = spec_size(h);
    const int nt = h->d.n_table + 1;
    CR_TRY(dalloc(h, &m.pos, (size_t)N));
    CR_TRY(dalloc(h, &m.q, (size_t)N));
    CR_TRY(dalloc(h, &m.phi, (size_t)N));
    CR_TRY(dalloc(h, &m.force, 3 * (size_t)N));
    CR_TRY(dalloc(h, &m.phiq, (size_t)nt));
    CR_TRY(dalloc(h, &m.gradphiq, (size_t)nt));
    CR_TRY(dalloc(h, &m.grid, (size_t)G));
    CR_TRY(dalloc(h, &m.spec, (size_t)S));
    CR_TRY(dalloc(h, &m.scale, (size_t)S));
    std::vector<R2> t1(nt), t2(nt);
    for (int i = 0; i < nt; ++i) {
        t1[i].x = (R)h->h_phiq[2 * i];
        t1[i].y = (R)h->h_phiq[2 * i + 1];
        t2[i].x = (R)h->h_gradphiq[2 * i];
        t2[i].y = (R)h->h_gradphiq[2 * i + 1];
    }
    CR_CUDA(h, cudaMemcpy(m.phiq, t1.data(), nt * sizeof(R2), cudaMemcpyHostToDevice));
    CR_CUDA(h, cudaMemcpy(m.gradphiq, t2.data(), nt * sizeof(R2), cudaMemcpyHostToDevice));
    scale_init_kernel<R><<<blocks_for(S, 256), 256>>>(m.scale, h->d.grid[0], h->d.grid[1], h->d.grid[2], h->L[0],
                                                       h->L[1], h->L[2], h->d.eta[0], h->d.eta[1], h->d.eta[2],
                                                       h->user.xi);
    CR_LAUNCH(h, "scale_init_kernel");
    CR_CUFFT(h, cufftPlan3d(&m.plan_fwd, h->d.grid[0], h->d.grid[1], h->d.grid[2], Prec<R>::kR2C));
    CR_CUFFT(h, cufftPlan3d(&m.plan_inv, h->d.grid[0], h->d.grid[1], h->d.grid[2], Prec<R>::kC2R));
    size_t s1 = spread_smem<R>(h), s2 = contract_smem<R>(h);
    if (s1 > 227 * 1024 || s2 > 227 * 1024)
        return fail(h, CR_BAD_PARAM, "support too large for the shared-memory tile buffer");
    int st = set_smem_attrs<R, 0>(h, s1, s2);
    if (st == CR_OK) st = set_smem_attrs<R, 9>(h, s1, s2);
    if (st == CR_OK) st = set_smem_attrs<R, 11>(h, s1, s2);
    if (st != CR_OK) return st;
    CR_CUDA(h, cudaDeviceSynchronize());
    m.ready = true;
    (void)sizeof(R4);
    (void)sizeof(C);
    return CR_OK;
}

template <typename R> void mesh_free(MeshBuffers<R> &m) {
    dfree(&m.pos);
    dfree(&m.q);
    dfree(&m.phi);
    dfree(&m.force);
    dfree(&m.phiq);
    dfree(&m.gradphiq);
    dfree(&m.grid);
    dfree(&m.spec);
    dfree(&m.scale);
    if (m.plan_fwd) cufftDestroy(m.plan_fwd);
    if (m.plan_inv) cufftDestroy(m.plan_inv);
    m.plan_fwd = m.plan_inv = 0;
    m.ready = false;
}

template <typename R> int cast_charges(cr_handle *h, MeshBuffers<R> &m, const double *d_q) {
    cast_kernel<R><<<blocks_for(h->N, 256), 256, 0, h->stream>>>(d_q, m.q, h->N);
    CR_LAUNCH(h, "cast_kernel");
    return CR_OK;
}

template <typename R> __global__ void to_double_kernel(const R *__restrict__ in, double *__restrict__ out, long n) {
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)in[i];
}

template <typename R> int cast_to_double(cr_handle *h, const R *in, double *out, long n) {
    if (n == 0) return CR_OK;
    to_double_kernel<R><<<blocks_for(n, 256), 256, 0, h->stream>>>(in, out, n);
    CR_LAUNCH(h, "to_double_kernel");
    return CR_OK;
}

template <typename R> int spread_only(cr_handle *h, MeshBuffers<R> &m) {
    ProfScope ps(h, PROF_SPREAD);
    const long G = grid_size(h);
    CR_CUDA(h, cudaMemsetAsync(m.grid, 0, G * sizeof(R), h->stream));
    CR_TRY(with_support<R>(h, [&](auto pt) -> int {
        constexpr int PT = decltype(pt)::value;
        if (PT == 0 || h->spread_mode == 1) {
            spread_tiles_kernel<R, PT><<<h->ntiles, 256, spread_smem<R>(h), h->stream>>>(
                m.pos, m.q, h->geo.wstart, h->geo.tile_start, h->geo.tile_beads, mesh_shape<R>(h),
                window_const<R>(h), (R)h->d.prefac, m.grid);
        } else {
            constexpr int BD = 8 + (PT ? PT : 1) - 1;
            spread_columns_kernel<R, (PT ? PT : 9)><<<h->ntiles, (BD * BD + 31) / 32 * 32, 0, h->stream>>>(
                m.pos, m.q, h->geo.wstart, h->geo.tile_start, h->geo.tile_beads, mesh_shape<R>(h),
                window_const<R>(h), (R)h->d.prefac, m.grid);
        }
        CR_LAUNCH(h, "spread kernel");
        return CR_OK;
    }));
    return CR_OK;
}

template <typename R> static int wave_mesh(cr_handle *h, MeshBuffers<R> &m) {
    CR_TRY(spread_only(h, m));
    CR_CUFFT(h, cufftSetStream(m.plan_fwd, h->stream));
    CR_CUFFT(h, cufftSetStream(m.plan_inv, h->stream));
    {
        ProfScope ps(h, PROF_FFT);
        CR_CUFFT(h, fft_forward(m.plan_fwd, m.grid, m.spec));
        ++h->fft_execs;
    }
    const int S = spec_size(h);
    {
        ProfScope ps(h, PROF_SCALE);
        scale_kernel<R, typename Prec<R>::C><<<blocks_for(S, 256), 256, 0, h->stream>>>(m.spec, m.scale, S);
        CR_LAUNCH(h, "scale_kernel");
    }
    {
        ProfScope ps(h, PROF_FFT);
        CR_CUFFT(h, fft_inverse(m.plan_inv, m.spec, m.grid));
        ++h->fft_execs;
    }
    return CR_OK;
}

template <typename R> int wave_potential(cr_handle *h, MeshBuffers<R> &m) {
    CR_TRY(wave_mesh(h, m));
    ProfScope ps(h, PROF_CONTRACT);
    CR_TRY(with_support<R>(h, [&](auto pt) -> int {
        contract_tiles_kernel<R, false, decltype(pt)::value><<<h->ntiles, 256, contract_smem<R>(h), h->stream>>>(
            m.pos, m.q, h->geo.wstart, h->geo.tile_start, h->geo.tile_beads, mesh_shape<R>(h), window_const<R>(h),
            (R)(h->d.quadW * h->d.prefac), m.grid, m.phi);
        CR_LAUNCH(h, "contract_tiles_kernel");
        return CR_OK;
    }));
    return CR_OK;
}

template <typename R> int wave_force(cr_handle *h, MeshBuffers<R> &m) {
    CR_TRY(wave_mesh(h, m));
    ProfScope ps(h, PROF_CONTRACT_FORCE);
    CR_TRY(with_support<R>(h, [&](auto pt) -> int {
        contract_tiles_kernel<R, true, decltype(pt)::value><<<h->ntiles, 256, contract_smem<R>(h), h->stream>>>(
            m.pos, m.q, h->geo.wstart, h->geo.tile_start, h->geo.tile_beads, mesh_shape<R>(h), window_const<R>(h),
            (R)(2.0 * h->d.quadW * h->d.prefac * h->d.xiterm), m.grid, m.force);
        CR_LAUNCH(h, "contract_force_tiles_kernel");
        return CR_OK;
    }));
    return CR_OK;
}

// Wave-space virial (FP64) of the charges already cast into m64.q: spread, forward
// transform, then the per-mode sums of wave_virial_kernel; out[0..5] the tensor (xx, xy,
// xz, yy, yz, zz), out[6] the wave energy.
int wave_virial(cr_handle *h, double *out) {
    MeshBuffers<double> &m = h->m64;
    CR_TRY(spread_only(h, m));
    CR_CUFFT(h, cufftSetStream(m.plan_fwd, h->stream));
    CR_CUFFT(h, fft_forward(m.plan_fwd, m.grid, m.spec));
    ++h->fft_execs;
    constexpr int kBlocks = 296;  // 2 per SM; partials summed in block order on the host
    std::vector<double> part((size_t)kBlocks * 7);
    double *d_part = nullptr;
    CR_TRY(dalloc(h, &d_part, part.size()));
    wave_virial_kernel<<<kBlocks, 256, 0, h->stream>>>(reinterpret_cast<const double2 *>(m.spec), m.scale,
                                                       h->d.grid[0], h->d.grid[1], h->d.grid[2], h->L[0], h->L[1],
                                                       h->L[2], h->user.xi, 0.5 * h->d.quadW, d_part);
    int st = check_cuda(h, cudaGetLastError(), "wave_virial_kernel");
    if (st == CR_OK) {
        ++h->launches;
        st = check_cuda(h, cudaMemcpyAsync(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                           h->stream), "wave virial partials");
    }
    if (st == CR_OK) st = check_cuda(h, cudaStreamSynchronize(h->stream), "wave virial");
    dfree(&d_part);
    if (st != CR_OK) return st;
    for (int c = 0; c < 7; ++c) out[c] = 0.0;
    for (int b = 0; b < kBlocks; ++b)
        for (int c = 0; c < 7; ++c) out[c] += part[(size_t)b * 7 + c];
    return CR_OK;
}

// Tile edge T for both precisions: tile counts, the shared-memory limits of the tile
// kernels, and the tile-sized geometry buffers (the geometry must be rebuilt after).
int mesh_set_tile(cr_handle *h, int T) {
    if (T < 2 || T > 32) return fail(h, CR_BAD_PARAM, "tile edge out of range");
    const int saved = h->tile;
    h->tile = T;
    const size_t s1f = spread_smem<float>(h), s2f = contract_smem<float>(h);
    const size_t s1d = spread_smem<double>(h), s2d = contract_smem<double>(h);
    if (std::max(std::max(s1f, s2f), std::max(s1d, s2d)) > 227 * 1024) {
        h->tile = saved;
        return fail(h, CR_BAD_PARAM, "tile edge too large for the shared-memory tile buffer");
    }
    h->ntiles = 1;
    for (int k = 0; k < 3; ++k) {
        h->ntiles_dim[k] = (h->d.grid[k] + T - 1) / T;
        h->ntiles *= h->ntiles_dim[k];
    }
    CR_TRY((set_smem_attrs<float, 0>(h, s1f, s2f)));
    CR_TRY((set_smem_attrs<double, 0>(h, s1d, s2d)));
    h->geo.valid = false;
    if (h->have_topology) CR_TRY(geometry_alloc(h));
    return CR_OK;
}

// ---- lockstep batches ----------------------------------------------------------------
// The mesh stages of a batched operator application: the same per-tile bodies as the
// single-system kernels, one CTA per (replica, tile) item, each replica's mesh and half
// spectrum in the batch buffers (replicas of one size consecutive, so that one batched
// cuFFT plan per size transforms them all).

namespace {

template <typename R> __device__ __forceinline__ MeshShape batch_shape(const BatchRep &b, int P) {
    MeshShape ms;
    for (int d = 0; d < 3; ++d) {
        ms.Ng[d] = b.Ng[d];
        ms.ntd[d] = b.ntd[d];
    }
    ms.T = 8;
    ms.P = P;
    ms.Bd = 8 + P - 1;
    ms.zp = sizeof(R) == 4 ? b.zp32 : b.zp64;
    return ms;
}

template <typename R> __device__ __forceinline__ WindowConst<R> batch_window(const BatchRep &b) {
    WindowConst<R> wc;
    for (int d = 0; d < 3; ++d) {
        wc.h[d] = (R)b.hm[d];
        wc.halfL[d] = (R)b.halfL[d];
        wc.inv_eta[d] = (R)b.inv_eta[d];
    }
    wc.xiterm = (R)b.xiterm;
    return wc;
}

template <typename R>
__global__ void cast_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items,
                                  const int *__restrict__ mask, int xin) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &b = reps[it.x];
    const double *in = b.vec[xin];
    R *out = brep_q<R>(b);
    for (int i = it.y * blockDim.x + threadIdx.x; i < b.N; i += b.vblk * blockDim.x) out[i] = (R)in[i];
}

// (the descriptor's addresses cost registers: bounded to the single kernel's four CTAs per SM)
template <typename R, int PT>
__global__ void __launch_bounds__(((8 + PT - 1) * (8 + PT - 1) + 31) / 32 * 32, sizeof(R) == 4 ? (PT == 9 ? 4 : 2) : 2)
    spread_batch_kernel(const BatchRep *__restrict__ reps, const int2 *__restrict__ items, const int *__restrict__ mask,
                        R *__restrict__ grid) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &b = reps[it.x];
    spread_columns_tile<R, PT>(it.y, brep_pos<R>(b), brep_q<R>(b), b.wstart, b.tile_start, b.tile_beads,
                               batch_shape<R>(b, PT), batch_window<R>(b), (R)b.prefac, grid + b.goff);
}

template <typename R, int PT>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 5 : 1) contract_batch_kernel(const BatchRep *__restrict__ reps,
                                                             const int2 *__restrict__ items,
                                                             const int *__restrict__ mask, const R *__restrict__ grid) {
    const int2 it = items[blockIdx.x];
    if (!mask[it.x]) return;
    const BatchRep &b = reps[it.x];
    contract_tile<R, false, PT>(it.y, brep_pos<R>(b), brep_q<R>(b), b.wstart, b.tile_start, b.tile_beads,
                                batch_shape<R>(b, PT), batch_window<R>(b), (R)b.coeff_phi, grid + b.goff,
                                brep_phi<R>(b));
}

// launch helpers: the batch's support selects the compiled kernels
template <typename R, typename F> int batch_with_support(cr_batch *bt, F f) {
    if (bt->support == 9) return f(std::integral_constant<int, 9>());
    if (bt->support == 11) return f(std::integral_constant<int, 11>());
    return batch_fail(bt, CR_BAD_PARAM, "lockstep batch: support must be 9 or 11");
}

// A failed batched transform: the cuFFT status, the group, and the stream's own state (an
// earlier asynchronous error shows there).
int batch_fft_fail(cr_batch *bt, cufftResult fr, const char *dir, size_t g, cudaStream_t s) {
    const cudaError_t q = cudaStreamQuery(s);
    const BatchFftGroup &G = bt->groups[g];
    return batch_fail(bt, CR_CUDA_ERROR,
                      std::string("batched ") + dir + " transform failed: cufftResult " + std::to_string((int)fr) +
                          ", size group " + std::to_string(g) + " (" + std::to_string(G.grid[0]) + "x" +
                          std::to_string(G.grid[1]) + "x" + std::to_string(G.grid[2]) + ", " +
                          std::to_string(G.reps.size()) + " replicas), stream: " + cudaGetErrorString(q));
}

template <typename R> R *batch_grid(cr_batch *bt);
template <> float *batch_grid<float>(cr_batch *bt) { return bt->grid32; }
template <> double *batch_grid<double>(cr_batch *bt) { return bt->grid64; }
template <typename R> typename Prec<R>::C *batch_spec(cr_batch *bt);
template <> cufftComplex *batch_spec<float>(cr_batch *bt) { return bt->spec32; }
template <> cufftDoubleComplex *batch_spec<double>(cr_batch *bt) { return bt->spec64; }
template <typename R> R *batch_scale(cr_batch *bt);
template <> float *batch_scale<float>(cr_batch *bt) { return bt->scale32; }
template <> double *batch_scale<double>(cr_batch *bt) { return bt->scale64; }

}  // namespace

// Contraction buffers of the batch (the same tile and support for every replica).
int batch_mesh_attrs(cr_batch *bt) {
    static size_t set32[2] = {0, 0}, set64[2] = {0, 0};
    std::lock_guard<std::mutex> lk(g_smem_mu);
    const int P = bt->support, Bd = 8 + P - 1;
    bt->contract_smem32 = ((size_t)Bd * Bd * contract_pitch(8, P, 4) + 8 * 6 * (size_t)P) * 4;
    bt->contract_smem64 = ((size_t)Bd * Bd * contract_pitch(8, P, 8) + 8 * 6 * (size_t)P) * 8;
    const int k = P == 9 ? 0 : 1;
    if (bt->contract_smem32 > set32[k]) {
        CR_TRY(batch_check(bt,
                           cudaFuncSetAttribute(P == 9 ? contract_batch_kernel<float, 9> : contract_batch_kernel<float, 11>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bt->contract_smem32),
                           "contract_batch_kernel attribute"));
        set32[k] = bt->contract_smem32;
    }
    if (bt->contract_smem64 > set64[k]) {
        CR_TRY(batch_check(bt,
                           cudaFuncSetAttribute(P == 9 ? contract_batch_kernel<double, 9>
                                                       : contract_batch_kernel<double, 11>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bt->contract_smem64),
                           "contract_batch_kernel attribute"));
        set64[k] = bt->contract_smem64;
    }
    return CR_OK;
}

template <typename R> int batch_cast(cr_batch *bt, const int *mask, int xin, cudaStream_t s) {
    if (bt->n_items[BL_VEC] == 0) return CR_OK;
    cast_batch_kernel<R><<<bt->n_items[BL_VEC], 256, 0, s>>>(bt->d_reps, bt->d_items[BL_VEC], mask, xin);
    ++bt->launches;
    return batch_check(bt, cudaGetLastError(), "cast_batch_kernel");
}

template <typename R>
int batch_wave(cr_batch *bt, const int *mask, const std::vector<char> &group_live, cudaStream_t s) {
    const int slot = sizeof(R) == 4 ? 1 : 0;
    R *grid = batch_grid<R>(bt);
    typename Prec<R>::C *spec = batch_spec<R>(bt);
    CR_TRY(batch_check(bt, cudaMemsetAsync(grid, 0, (size_t)bt->G * sizeof(R), s), "batch mesh clear"));
    const int nt = bt->n_items[BL_TILES];
    CR_TRY(batch_with_support<R>(bt, [&](auto pt) -> int {
        constexpr int PT = decltype(pt)::value;
        constexpr int BD = 8 + PT - 1;
        if (nt > 0) {
            spread_batch_kernel<R, PT><<<nt, (BD * BD + 31) / 32 * 32, 0, s>>>(bt->d_reps, bt->d_items[BL_TILES], mask,
                                                                              grid);
            ++bt->launches;
            CR_TRY(batch_check(bt, cudaGetLastError(), "spread_batch_kernel"));
        }
        return CR_OK;
    }));
    for (size_t g = 0; g < bt->groups.size(); ++g) {
        if (!group_live[g]) continue;
        BatchFftGroup &G = bt->groups[g];
        cufftResult fr = cufftSetStream(G.fwd[slot], s);
        if (fr == CUFFT_SUCCESS) fr = fft_forward(G.fwd[slot], grid + G.goff, spec + G.soff);
        if (fr != CUFFT_SUCCESS) return batch_fft_fail(bt, fr, "forward", g, s);
        ++bt->fft_execs;
    }
    const long long S = bt->S;
    if (S > 0) {
        scale_kernel<R, typename Prec<R>::C><<<blocks_for(S, 256), 256, 0, s>>>(spec, batch_scale<R>(bt), (int)S);
        ++bt->launches;
        CR_TRY(batch_check(bt, cudaGetLastError(), "scale_kernel (batch)"));
    }
    for (size_t g = 0; g < bt->groups.size(); ++g) {
        if (!group_live[g]) continue;
        BatchFftGroup &G = bt->groups[g];
        cufftResult fr = cufftSetStream(G.inv[slot], s);
        if (fr == CUFFT_SUCCESS) fr = fft_inverse(G.inv[slot], spec + G.soff, grid + G.goff);
        if (fr != CUFFT_SUCCESS) return batch_fft_fail(bt, fr, "inverse", g, s);
        ++bt->fft_execs;
    }
    return batch_with_support<R>(bt, [&](auto pt) -> int {
        constexpr int PT = decltype(pt)::value;
        if (nt > 0) {
            contract_batch_kernel<R, PT><<<nt, 256, sizeof(R) == 4 ? bt->contract_smem32 : bt->contract_smem64, s>>>(
                bt->d_reps, bt->d_items[BL_TILES], mask, grid);
            ++bt->launches;
            CR_TRY(batch_check(bt, cudaGetLastError(), "contract_batch_kernel"));
        }
        return CR_OK;
    });
}

template int batch_cast<float>(cr_batch *, const int *, int, cudaStream_t);
template int batch_cast<double>(cr_batch *, const int *, int, cudaStream_t);
template int batch_wave<float>(cr_batch *, const int *, const std::vector<char> &, cudaStream_t);
template int batch_wave<double>(cr_batch *, const int *, const std::vector<char> &, cudaStream_t);

template int mesh_init<float>(cr_handle *, MeshBuffers<float> &);
template int mesh_init<double>(cr_handle *, MeshBuffers<double> &);
template void mesh_free<float>(MeshBuffers<float> &);
template void mesh_free<double>(MeshBuffers<double> &);
template int cast_charges<float>(cr_handle *, MeshBuffers<float> &, const double *);
template int cast_charges<double>(cr_handle *, MeshBuffers<double> &, const double *);
template int cast_to_double<float>(cr_handle *, const float *, double *, long);
template int cast_to_double<double>(cr_handle *, const double *, double *, long);
template int spread_only<float>(cr_handle *, MeshBuffers<float> &);
template int spread_only<double>(cr_handle *, MeshBuffers<double> &);
template int wave_potential<float>(cr_handle *, MeshBuffers<float> &);
template int wave_potential<double>(cr_handle *, MeshBuffers<double> &);
template int wave_force<float>(cr_handle *, MeshBuffers<float> &);
template int wave_force<double>(cr_handle *, MeshBuffers<double> &);

}  // namespace cr
