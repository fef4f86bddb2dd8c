// noalloc.cu -- Gaussian spreading of charges onto the mesh without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need the charge
// mesh: a host engine that owns all device memory through its own pool (an MD code's
// array manager) and forbids allocations behind its back, or a time-step loop where a
// cudaMalloc/cudaFree would synchronise the whole device while other streams are busy.
// cr_spread_noalloc serves them: it does the same spreading as cr_spread in FP64
// (ConductorRigid.cu:144-234, with the window rule of :207-210), but keeps its scratch
// (per-bead window starts and the bead-to-tile binning) in one file-scope device array
// of fixed size instead of allocating it.  The caller passes the positions, charges and
// the output mesh.
//
// The array lives in every GPU that loads this library until the process exits
// (CR_NOALLOC_SCRATCH_BYTES).  Host code cannot use the array's name as a device
// address, so each device's address is looked up once with cudaGetSymbolAddress,
// with that device current, on the first call made on that device.  All calls share
// the one array and it keeps the last call's contents; every call clears what must
// start from zero.  Calls that overlap on the GPU (two streams, or two threads) race on
// the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/conductor_rigid.h"

namespace {

constexpr int kTile = 8;       // spreading tile edge in mesh nodes (as cr_spread)
constexpr int kMaxSupport = 16;
constexpr double kPi = 3.14159265358979323846;

// Layout of the scratch array.
constexpr size_t kOffWstart = 0;                                                        // int4[MAX_BEADS]
constexpr size_t kOffBeads = kOffWstart + sizeof(int4) * CR_NOALLOC_MAX_BEADS;          // int[MAX_BEADS]
constexpr size_t kOffCount = kOffBeads + sizeof(int) * CR_NOALLOC_MAX_BEADS;            // int[MAX_TILES+1]
constexpr size_t kOffStart = kOffCount + sizeof(int) * (CR_NOALLOC_MAX_TILES + 1);      // int[MAX_TILES+1]
constexpr size_t kOffCursor = kOffStart + sizeof(int) * (CR_NOALLOC_MAX_TILES + 1);     // int[MAX_TILES]
constexpr size_t kOffFlag = kOffCursor + sizeof(int) * CR_NOALLOC_MAX_TILES;            // int
constexpr size_t kScratchBytes = kOffFlag + 256;
static_assert(kScratchBytes <= CR_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the declared size");

__device__ __align__(256) unsigned char g_spread_scratch[CR_NOALLOC_SCRATCH_BYTES];

std::mutex g_mutex;
void *g_scratch_addr[64] = {nullptr};
thread_local std::string g_error;

int set_error(int status, const char *msg) {
    g_error = msg;
    return status;
}

// Device address of the scratch array on the current device (looked up once).
int scratch_address(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(CR_CUDA_ERROR, "cudaGetDevice failed");
    }
    if (dev < 0 || dev >= 64) return set_error(CR_BAD_PARAM, "device index above 63");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_spread_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return set_error(CR_CUDA_ERROR, "cudaGetSymbolAddress of the spreading scratch failed");
        }
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_addr[dev]);
    return CR_OK;
}

struct Shape {
    int N[3];
    int ntd[3];
    int P, Bd;
    double L[3], h[3], inv_eta[3];
    double xiterm, prefac;
};

__device__ __forceinline__ int wrapmod(int s, int n) {
    int r = s % n;
    return r < 0 ? r + n : r;
}

// Wrapped position and first window node per dimension, in the same FP64 operation
// order as cr_spread (round-to-nearest intrinsics, no fused multiply-add).
__global__ void noalloc_bin_kernel(int n, const double *__restrict__ pos, Shape s, int4 *wstart, int *count,
                                   int *flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int st[3], t[3];
    for (int d = 0; d < 3; ++d) {
        double v = pos[3 * (size_t)i + d];
        if (!isfinite(v) || fabs(v) > 1e6 * s.L[d]) {
            atomicOr(flag, 1);
            v = 0.0;
        }
        const double f = floor(__ddiv_rn(__dadd_rn(v, 0.5 * s.L[d]), s.L[d]));
        double x = f == 0.0 ? v : __dsub_rn(v, __dmul_rn(s.L[d], f));
        x = fmin(fmax(x, -0.5 * s.L[d]), 0.5 * s.L[d]);
        const double frac = __ddiv_rn(__dadd_rn(x, 0.5 * s.L[d]), s.L[d]);
        const double u = __dmul_rn(frac, (double)s.N[d]);
        const int x0 = (int)u;
        st[d] = x0 - s.P / 2 + 1 - (s.P & 1) * (__dsub_rn(u, (double)x0) < 0.5 ? 1 : 0);
        t[d] = wrapmod(st[d], s.N[d]) / kTile;
    }
    const int tile = (t[0] * s.ntd[1] + t[1]) * s.ntd[2] + t[2];
    wstart[i] = make_int4(st[0], st[1], st[2], tile);
    atomicAdd(count + tile, 1);
}

// Exclusive scan of count[0..n) into start[0..n] and cursor[0..n) by one CTA.
__global__ void noalloc_scan_kernel(int n, const int *__restrict__ count, int *start, int *cursor) {
    __shared__ int carry;
    __shared__ int warp_tot[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < n ? count[i] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const int nw = blockDim.x >> 5;
            int wv = lane < nw ? warp_tot[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, wv, o);
                if (lane >= o) wv += y;
            }
            if (lane < nw) warp_tot[lane] = wv;
        }
        __syncthreads();
        const int before = carry + (warp > 0 ? warp_tot[warp - 1] : 0) + incl - v;
        if (i < n) {
            start[i] = before;
            cursor[i] = before;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) start[n] = carry;
}

__global__ void noalloc_scatter_kernel(int n, const int4 *__restrict__ wstart, int *cursor, int *beads) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    beads[atomicAdd(cursor + wstart[i].w, 1)] = i;
}

// One CTA per tile: accumulate the tile's beads in a (T+P-1)^3 shared buffer, then add
// the buffer to the mesh (the algorithm of cr_spread, positions read from the caller).
__global__ void __launch_bounds__(256) noalloc_spread_kernel(const double *__restrict__ pos,
                                                             const double *__restrict__ q,
                                                             const int4 *__restrict__ wstart,
                                                             const int *__restrict__ tile_start,
                                                             const int *__restrict__ tile_beads, Shape s,
                                                             double *__restrict__ grid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *buf = reinterpret_cast<double *>(smem_raw);
    const int Bd = s.Bd, P = s.P;
    const int nbuf = Bd * Bd * Bd;
    const int tile = blockIdx.x;
    const int b0 = tile_start[tile], b1 = tile_start[tile + 1];
    if (b0 == b1) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    double *w = buf + nbuf + warp * 3 * P;
    for (int i = threadIdx.x; i < nbuf; i += blockDim.x) buf[i] = 0.0;
    __syncthreads();
    const int tz = tile % s.ntd[2], ty = (tile / s.ntd[2]) % s.ntd[1], tx = tile / (s.ntd[2] * s.ntd[1]);
    for (int k = b0 + warp; k < b1; k += nw) {
        const int i = tile_beads[k];
        const int4 st = wstart[i];
        double x[3];
        for (int d = 0; d < 3; ++d) {
            double v = pos[3 * (size_t)i + d];
            if (!isfinite(v)) v = 0.0;
            const double f = floor(__ddiv_rn(__dadd_rn(v, 0.5 * s.L[d]), s.L[d]));
            x[d] = f == 0.0 ? v : __dsub_rn(v, __dmul_rn(s.L[d], f));
            x[d] = fmin(fmax(x[d], -0.5 * s.L[d]), 0.5 * s.L[d]);
        }
        for (int t = lane; t < 3 * P; t += 32) {
            const int d = t >= 2 * P ? 2 : (t >= P ? 1 : 0);
            const int tt = t - d * P;
            const int sd = d == 0 ? st.x : (d == 1 ? st.y : st.z);
            const double r = s.h[d] * (double)(sd + tt) - 0.5 * s.L[d] - x[d];
            w[t] = exp(-s.xiterm * r * r * s.inv_eta[d]);
        }
        __syncwarp();
        const int ox = wrapmod(st.x, s.N[0]) - tx * kTile;
        const int oy = wrapmod(st.y, s.N[1]) - ty * kTile;
        const int oz = wrapmod(st.z, s.N[2]) - tz * kTile;
        const double c = s.prefac * q[i];
        if (ox >= 0 && ox < kTile && oy >= 0 && oy < kTile && oz >= 0 && oz < kTile) {
            for (int e = lane; e < P * P; e += 32) {
                const int b = e / P, cc = e - b * P;
                const double wyz = c * w[P + b] * w[2 * P + cc];
                double *col = buf + ((size_t)ox * Bd + (oy + b)) * Bd + (oz + cc);
                for (int a = 0; a < P; ++a) atomicAdd(col + (size_t)a * Bd * Bd, wyz * w[a]);
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int n = threadIdx.x; n < nbuf; n += blockDim.x) {
        const double v = buf[n];
        if (v == 0.0) continue;
        const int bz = n % Bd, by = (n / Bd) % Bd, bx = n / (Bd * Bd);
        const int gx = (tx * kTile + bx) % s.N[0];
        const int gy = (ty * kTile + by) % s.N[1];
        const int gz = (tz * kTile + bz) % s.N[2];
        atomicAdd(grid + ((size_t)gx * s.N[1] + gy) * s.N[2] + gz, v);
    }
}

int cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return CR_OK;
    cudaGetLastError();
    g_error = std::string(what) + ": " + cudaGetErrorString(e);
    return CR_CUDA_ERROR;
}

}  // namespace

extern "C" {

const char *cr_noalloc_last_error(void) { return g_error.c_str(); }

int cr_spread_noalloc(const cr_derived *d, double xi, const double L[3], int n_beads, const double *d_pos,
                      const double *d_q, double *d_grid, void *stream) {
    g_error.clear();
    if (!d || !L || !d_grid || n_beads < 0 || (n_beads > 0 && (!d_pos || !d_q)))
        return set_error(CR_BAD_PARAM, "null argument or negative bead count");
    if (n_beads > CR_NOALLOC_MAX_BEADS)
        return set_error(CR_BAD_PARAM, "cr_spread_noalloc: more beads than CR_NOALLOC_MAX_BEADS");
    Shape s;
    long ntiles = 1;
    for (int k = 0; k < 3; ++k) {
        if (d->grid[k] < 1 || !(L[k] > 0) || !(d->h[k] > 0) || !(d->eta[k] > 0))
            return set_error(CR_BAD_PARAM, "invalid mesh or box");
        s.N[k] = d->grid[k];
        s.ntd[k] = (d->grid[k] + kTile - 1) / kTile;
        ntiles *= s.ntd[k];
        s.L[k] = L[k];
        s.h[k] = d->h[k];
        s.inv_eta[k] = 1.0 / d->eta[k];
    }
    if (ntiles > CR_NOALLOC_MAX_TILES)
        return set_error(CR_BAD_PARAM, "cr_spread_noalloc: mesh needs more tiles than CR_NOALLOC_MAX_TILES");
    if (d->support < 1 || d->support > kMaxSupport || d->support > d->grid[0] || d->support > d->grid[1] ||
        d->support > d->grid[2])
        return set_error(CR_BAD_PARAM, "cr_spread_noalloc: support outside 1..16 or above the mesh size");
    if (!(xi > 0)) return set_error(CR_BAD_PARAM, "xi must be positive");
    s.P = d->support;
    s.Bd = kTile + s.P - 1;
    s.xiterm = 2.0 * xi * xi;
    s.prefac = s.xiterm * xi / kPi * std::sqrt(2.0 / (kPi * d->eta[0] * d->eta[1] * d->eta[2]));
    unsigned char *base = nullptr;
    int st = scratch_address(&base);
    if (st != CR_OK) return st;
    int4 *wstart = reinterpret_cast<int4 *>(base + kOffWstart);
    int *beads = reinterpret_cast<int *>(base + kOffBeads);
    int *count = reinterpret_cast<int *>(base + kOffCount);
    int *start = reinterpret_cast<int *>(base + kOffStart);
    int *cursor = reinterpret_cast<int *>(base + kOffCursor);
    int *flag = reinterpret_cast<int *>(base + kOffFlag);
    cudaStream_t strm = static_cast<cudaStream_t>(stream);
    const size_t G = (size_t)s.N[0] * s.N[1] * s.N[2];
    if ((st = cuda_status(cudaMemsetAsync(d_grid, 0, G * sizeof(double), strm), "clear mesh")) != CR_OK) return st;
    if (n_beads == 0) return cuda_status(cudaStreamSynchronize(strm), "cr_spread_noalloc");
    if ((st = cuda_status(cudaMemsetAsync(count, 0, sizeof(int) * (ntiles + 1), strm), "clear counts")) != CR_OK)
        return st;
    if ((st = cuda_status(cudaMemsetAsync(flag, 0, sizeof(int), strm), "clear flag")) != CR_OK) return st;
    const int nb = (n_beads + 255) / 256;
    noalloc_bin_kernel<<<nb, 256, 0, strm>>>(n_beads, d_pos, s, wstart, count, flag);
    if ((st = cuda_status(cudaGetLastError(), "noalloc_bin_kernel")) != CR_OK) return st;
    int bad = 0;
    if ((st = cuda_status(cudaMemcpyAsync(&bad, flag, sizeof(int), cudaMemcpyDeviceToHost, strm), "read flag")) !=
        CR_OK)
        return st;
    if ((st = cuda_status(cudaStreamSynchronize(strm), "cr_spread_noalloc")) != CR_OK) return st;
    if (bad) return set_error(CR_NUMERICAL, "non-finite or out-of-range bead position");
    noalloc_scan_kernel<<<1, 1024, 0, strm>>>((int)ntiles, count, start, cursor);
    if ((st = cuda_status(cudaGetLastError(), "noalloc_scan_kernel")) != CR_OK) return st;
    noalloc_scatter_kernel<<<nb, 256, 0, strm>>>(n_beads, wstart, cursor, beads);
    if ((st = cuda_status(cudaGetLastError(), "noalloc_scatter_kernel")) != CR_OK) return st;
    const size_t smem = ((size_t)s.Bd * s.Bd * s.Bd + 8 * 3 * (size_t)s.P) * sizeof(double);
    if ((st = cuda_status(cudaFuncSetAttribute(noalloc_spread_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem),
                          "shared memory attribute")) != CR_OK)
        return st;
    noalloc_spread_kernel<<<(unsigned)ntiles, 256, smem, strm>>>(d_pos, d_q, wstart, start, beads, s, d_grid);
    if ((st = cuda_status(cudaGetLastError(), "noalloc_spread_kernel")) != CR_OK) return st;
    return cuda_status(cudaStreamSynchronize(strm), "cr_spread_noalloc");
}

}  // extern "C"
