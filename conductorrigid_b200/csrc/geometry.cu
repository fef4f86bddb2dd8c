// geometry.cu -- per-solve geometry: wrapped positions, spreading windows, tile bins,
// cell list and the full neighbour list within the real-space cutoff.
//
// Positions are fixed during one solve, so everything here runs once per solve and the
// operator kernels reuse it for every GMRES iteration.  All binning is a stable radix
// sort of (key, bead index) pairs, so every list is ordered by bead index within a bin
// and identical from run to run.
//
// The spreading window start follows ConductorRigid.cu:193-210 in FP64 with explicit
// round-to-nearest intrinsics (no fused multiply-add), the same operation sequence as
// the host oracle, so window indices are bit-identical on both sides.  Pair distances
// in the neighbour-list builder use dx -= L*rint(dx*(1/L)) and d2 = dx*dx + dy*dy + dz*dz
// the same way; the resulting pair set is the one HOOMD's NeighborListGPUBinned gives
// the reference (compute.py:38-44, no exclusions, both directions).
#include <cub/cub.cuh>

#include <algorithm>

#include "cr_internal.cuh"

namespace cr {

namespace {

struct CellGrid {
    int nc[3];
    int k;          // stencil half width in cells (0: all pairs)
    double L[3], Linv[3];
};

__device__ __forceinline__ int wrapmod(int s, int n) {
    int r = s % n;
    return r < 0 ? r + n : r;
}

__device__ __forceinline__ double min_image(double dx, double L, double Linv) {
    const double img = rint(__dmul_rn(dx, Linv));
    return __dsub_rn(dx, __dmul_rn(L, img));
}

__device__ __forceinline__ double pair_d2(double4 a, double4 b, const CellGrid &cg) {
    const double dx = min_image(__dsub_rn(a.x, b.x), cg.L[0], cg.Linv[0]);
    const double dy = min_image(__dsub_rn(a.y, b.y), cg.L[1], cg.Linv[1]);
    const double dz = min_image(__dsub_rn(a.z, b.z), cg.L[2], cg.Linv[2]);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// First node of the P-point window along one dimension (ConductorRigid.cu:193-210).
__device__ __forceinline__ int window_start(double x, double L, int N, int P) {
    const double frac = __ddiv_rn(__dadd_rn(x, 0.5 * L), L);
    const double u = __dmul_rn(frac, (double)N);
    const int x0 = (int)u;
    return x0 - P / 2 + 1 - (P & 1) * (__dsub_rn(u, (double)x0) < 0.5 ? 1 : 0);
}

struct PrepArgs {
    int N;
    double L[3];
    int Ng[3];
    int P, T;
    int ntd[3];
    CellGrid cg;
};

// Non-finite inputs are flagged in *bad and replaced by 0 so that no index below is
// ever computed from them; the host turns the flag into CR_NUMERICAL.
__global__ void prepare_kernel(PrepArgs a, const double *__restrict__ pos_in, double4 *pos64, float4 *pos32,
                               int4 *wstart, int *tile_key, int *cell_key, int *iota, int *bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    double x[3];
    int s[3], t[3], c[3];
    for (int d = 0; d < 3; ++d) {
        double v = pos_in[3 * (size_t)i + d];
        if (!isfinite(v) || fabs(v) > 1e6 * a.L[d]) {
            atomicOr(bad, 1);
            v = 0.0;
        }
        // wrap into [-L/2, L/2) (a no-op for positions already in the box)
        const double f = floor(__ddiv_rn(__dadd_rn(v, 0.5 * a.L[d]), a.L[d]));
        x[d] = f == 0.0 ? v : __dsub_rn(v, __dmul_rn(a.L[d], f));
        x[d] = fmin(fmax(x[d], -0.5 * a.L[d]), 0.5 * a.L[d]);
        s[d] = window_start(x[d], a.L[d], a.Ng[d], a.P);
        t[d] = wrapmod(s[d], a.Ng[d]) / a.T;
        int cc = (int)floor(__ddiv_rn(__dadd_rn(x[d], 0.5 * a.L[d]), a.L[d]) * a.cg.nc[d]);
        c[d] = min(max(cc, 0), a.cg.nc[d] - 1);
    }
    pos64[i] = make_double4(x[0], x[1], x[2], 0.0);
    pos32[i] = make_float4((float)x[0], (float)x[1], (float)x[2], 0.f);
    const int tile = (t[0] * a.ntd[1] + t[1]) * a.ntd[2] + t[2];
    wstart[i] = make_int4(s[0], s[1], s[2], tile);
    tile_key[i] = tile;
    cell_key[i] = (c[0] * a.cg.nc[1] + c[1]) * a.cg.nc[2] + c[2];
    iota[i] = i;
}

__global__ void histogram_kernel(const int *__restrict__ key, int n, int *count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(count + key[i], 1);
}

struct ToI64 {
    __host__ __device__ int64_t operator()(int v) const { return (int64_t)v; }
};

// Visit the candidate beads of bead i: the (2k+1)^3 cell stencil around its cell, or
// every bead when the box holds fewer than 2k+1 cells per dimension (k == 0).
template <typename F>
__device__ __forceinline__ void for_each_candidate(int i, int N, const CellGrid &cg, const int *cell_of,
                                                   const int *cell_start, const int *cell_beads, int lane, F f) {
    if (cg.k == 0) {
        for (int base = 0; base < N; base += 32) {
            const int j = base + lane;
            f(j < N ? j : -1);
        }
        return;
    }
    const int ci = cell_of[i];
    const int cz = ci % cg.nc[2], cy = (ci / cg.nc[2]) % cg.nc[1], cx = ci / (cg.nc[2] * cg.nc[1]);
    for (int a = -cg.k; a <= cg.k; ++a)
        for (int b = -cg.k; b <= cg.k; ++b)
            for (int c = -cg.k; c <= cg.k; ++c) {
                const int x = wrapmod(cx + a, cg.nc[0]), y = wrapmod(cy + b, cg.nc[1]), z = wrapmod(cz + c, cg.nc[2]);
                const int cell = (x * cg.nc[1] + y) * cg.nc[2] + z;
                const int m0 = cell_start[cell], m1 = cell_start[cell + 1];
                for (int base = m0; base < m1; base += 32) {
                    const int m = base + lane;
                    f(m < m1 ? cell_beads[m] : -1);
                }
            }
}

__global__ void nlist_count_kernel(int N, const double4 *__restrict__ pos, CellGrid cg, double rl2,
                                   const int *__restrict__ cell_of, const int *__restrict__ cell_start,
                                   const int *__restrict__ cell_beads, int *count) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    const double4 pi = pos[i];
    int cnt = 0;
    for_each_candidate(i, N, cg, cell_of, cell_start, cell_beads, lane, [&](int j) {
        if (j >= 0 && j != i && pair_d2(pi, pos[j], cg) < rl2) ++cnt;
    });
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) count[i] = cnt;
}

__global__ void nlist_fill_kernel(int N, const double4 *__restrict__ pos, CellGrid cg, double rl2,
                                  const int *__restrict__ cell_of, const int *__restrict__ cell_start,
                                  const int *__restrict__ cell_beads, const int64_t *__restrict__ head,
                                  const int *__restrict__ count, int *list, int64_t capacity) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    const double4 pi = pos[i];
    const int64_t h0 = head[i];
    const int limit = count[i];
    int filled = 0;
    for_each_candidate(i, N, cg, cell_of, cell_start, cell_beads, lane, [&](int j) {
        const bool hit = j >= 0 && j != i && pair_d2(pi, pos[j], cg) < rl2;
        const unsigned mask = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const int slot = filled + __popc(mask & ((1u << lane) - 1u));
            const int64_t at = h0 + slot;
            if (slot < limit && at < capacity) list[at] = j;
        }
        filled += __popc(mask);
    });
}

CellGrid make_cell_grid(const cr_handle *h, double r_list) {
    CellGrid cg;
    for (int d = 0; d < 3; ++d) {
        cg.L[d] = h->L[d];
        cg.Linv[d] = 1.0 / h->L[d];
    }
    // half-width cells with a 5^3 stencil when the box is large enough, full-width
    // cells with a 3^3 stencil otherwise, all pairs for tiny boxes
    cg.k = 0;
    for (int k = 2; k >= 1; --k) {
        bool ok = true;
        int nc[3];
        for (int d = 0; d < 3; ++d) {
            nc[d] = (int)std::floor(h->L[d] / (r_list / k));
            if (nc[d] < 2 * k + 1) ok = false;
        }
        if (ok) {
            cg.k = k;
            for (int d = 0; d < 3; ++d) cg.nc[d] = nc[d];
            break;
        }
    }
    if (cg.k == 0)
        for (int d = 0; d < 3; ++d) cg.nc[d] = 1;
    return cg;
}

}  // namespace

int geometry_alloc(cr_handle *h) {
    Geometry &g = h->geo;
    const int N = h->N;
    CR_TRY(dalloc(h, &h->d_flag, 1));
    CR_TRY(dalloc(h, &g.wstart, (size_t)N));
    CR_TRY(dalloc(h, &g.tile_start, (size_t)h->ntiles + 1));
    CR_TRY(dalloc(h, &g.tile_count, (size_t)h->ntiles + 1));
    CR_TRY(dalloc(h, &g.tile_beads, (size_t)N));
    CR_TRY(dalloc(h, &g.nl_count, (size_t)N));
    CR_TRY(dalloc(h, &g.nl_head, (size_t)N));
    CR_TRY(dalloc(h, &g.cell_of, (size_t)N));
    CR_TRY(dalloc(h, &g.cell_beads, (size_t)N));
    CR_TRY(dalloc(h, &h->d_keys, (size_t)N));
    CR_TRY(dalloc(h, &h->d_keys_alt, (size_t)N));
    CR_TRY(dalloc(h, &h->d_vals, (size_t)N));
    CR_TRY(dalloc(h, &h->d_vals_alt, (size_t)N));
    CR_TRY(realspace_alloc(h));
    // CUB scratch: the largest of the sorts and scans used here
    size_t b1 = 0, b2 = 0, b3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b1, h->d_keys, h->d_keys_alt, h->d_vals, h->d_vals_alt, N);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, g.tile_count, g.tile_start, std::max(h->ntiles + 1, N + 1));
    cub::TransformInputIterator<int64_t, ToI64, const int *> it(g.nl_count, ToI64());
    cub::DeviceScan::ExclusiveSum(nullptr, b3, it, g.nl_head, N);
    size_t b4 = 0;
    {
        long long *lh = nullptr;
        cub::DeviceScan::ExclusiveSum(nullptr, b4, g.tile_count, lh, N + 1);
    }
    size_t need = std::max(std::max(b1, b4), std::max(b2, b3)) + 256;
    if (need > h->sort_tmp_bytes) {
        dfree(reinterpret_cast<char **>(&h->d_sort_tmp));
        CR_TRY(dalloc(h, reinterpret_cast<char **>(&h->d_sort_tmp), need));
        h->sort_tmp_bytes = need;
    }
    g.valid = false;
    return CR_OK;
}

void geometry_free(cr_handle *h) {
    Geometry &g = h->geo;
    dfree(&h->d_flag);
    dfree(&g.wstart);
    dfree(&g.tile_start);
    dfree(&g.tile_count);
    dfree(&g.tile_beads);
    dfree(&g.nl_count);
    dfree(&g.nl_head);
    dfree(&g.nl_list);
    dfree(&g.cell_of);
    dfree(&g.cell_start);
    dfree(&g.cell_beads);
    g.nl_capacity = 0;
    g.ncell_alloc = 0;
    g.valid = false;
    dfree(&h->d_keys);
    dfree(&h->d_keys_alt);
    dfree(&h->d_vals);
    dfree(&h->d_vals_alt);
    realspace_free(h);
    dfree(reinterpret_cast<char **>(&h->d_sort_tmp));
    h->sort_tmp_bytes = 0;
}

// Stable counting sort of beads by key: sorted values into `sorted`, bin starts into
// `start[0..nbins]`.
static int bin_beads(cr_handle *h, const int *key, int nbins, int *count, int *start, int *sorted) {
    const int N = h->N;
    cudaStream_t s = h->stream;
    CR_CUDA(h, cudaMemsetAsync(count, 0, (size_t)(nbins + 1) * sizeof(int), s));
    histogram_kernel<<<blocks_for(N, 256), 256, 0, s>>>(key, N, count);
    CR_LAUNCH(h, "histogram_kernel");
    size_t bytes = h->sort_tmp_bytes;
    CR_CUDA(h, cub::DeviceScan::ExclusiveSum(h->d_sort_tmp, bytes, count, start, nbins + 1, s));
    bytes = h->sort_tmp_bytes;
    CR_CUDA(h, cub::DeviceRadixSort::SortPairs(h->d_sort_tmp, bytes, key, h->d_keys_alt, h->d_vals, sorted, N, 0,
                                               32, s));
    return CR_OK;
}

static int build_list(cr_handle *h, const CellGrid &cg, const int *cell_of, const int *cell_start,
                      const int *cell_beads, double r_list, int *count, int64_t *head, int **list, int64_t *capacity,
                      int64_t *total, bool grow) {
    const int N = h->N;
    cudaStream_t s = h->stream;
    const double rl2 = r_list * r_list;
    const int threads = 256;
    const int blocks = blocks_for((long)N * 32, threads);
    nlist_count_kernel<<<blocks, threads, 0, s>>>(N, h->m64.pos, cg, rl2, cell_of, cell_start, cell_beads, count);
    CR_LAUNCH(h, "nlist_count_kernel");
    cub::TransformInputIterator<int64_t, ToI64, const int *> it(count, ToI64());
    size_t bytes = h->sort_tmp_bytes;
    CR_CUDA(h, cub::DeviceScan::ExclusiveSum(h->d_sort_tmp, bytes, it, head, N, s));
    int64_t last_head = 0;
    int last_count = 0;
    if (N > 0) {
        CR_CUDA(h, cudaMemcpyAsync(&last_head, head + N - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        CR_CUDA(h, cudaMemcpyAsync(&last_count, count + N - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    CR_CUDA(h, cudaStreamSynchronize(s));
    *total = last_head + last_count;
    if (grow && *total > *capacity) {
        int64_t cap = *total + *total / 8 + 1024;
        CR_TRY(dalloc(h, list, (size_t)cap));
        *capacity = cap;
    }
    if (*list && *capacity > 0 && N > 0) {
        nlist_fill_kernel<<<blocks, threads, 0, s>>>(N, h->m64.pos, cg, rl2, cell_of, cell_start, cell_beads, head,
                                                     count, *list, *capacity);
        CR_LAUNCH(h, "nlist_fill_kernel");
    }
    return CR_OK;
}

__global__ void cell_key_kernel(int N, const double4 *__restrict__ pos, CellGrid cg, int *key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double4 p = pos[i];
    const double x[3] = {p.x, p.y, p.z};
    int c[3];
    for (int d = 0; d < 3; ++d) {
        int cc = (int)floor(__ddiv_rn(__dadd_rn(x[d], 0.5 * cg.L[d]), cg.L[d]) * cg.nc[d]);
        c[d] = min(max(cc, 0), cg.nc[d] - 1);
    }
    key[i] = (c[0] * cg.nc[1] + c[1]) * cg.nc[2] + c[2];
}

__global__ void segment_end_kernel(int N, const int64_t *head, const int *count, int64_t *end) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) end[i] = head[i] + count[i];
}

// Cell list of the current positions for cell grid cg: cell_of[N] keys, start[ncell+1],
// beads[N] (ascending bead index within a cell).
static int cell_bins(cr_handle *h, const CellGrid &cg, int *cell_of, int **start, size_t *start_alloc,
                     int *beads) {
    const int N = h->N;
    const size_t ncell = (size_t)cg.nc[0] * cg.nc[1] * cg.nc[2];
    if (ncell + 1 > *start_alloc) {
        CR_TRY(dalloc(h, start, ncell + 1));
        *start_alloc = ncell + 1;
    }
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, *start, *start, (int)ncell + 1);
    if (b + 256 > h->sort_tmp_bytes) {
        dfree(reinterpret_cast<char **>(&h->d_sort_tmp));
        CR_TRY(dalloc(h, reinterpret_cast<char **>(&h->d_sort_tmp), b + 256));
        h->sort_tmp_bytes = b + 256;
    }
    cell_key_kernel<<<blocks_for(N, 256), 256, 0, h->stream>>>(N, h->m64.pos, cg, cell_of);
    CR_LAUNCH(h, "cell_key_kernel");
    int *count = nullptr;
    CR_TRY(dalloc(h, &count, ncell + 1));
    int st = bin_beads(h, cell_of, (int)ncell, count, *start, beads);
    cudaStreamSynchronize(h->stream);
    dfree(&count);
    return st;
}

int geometry_update(cr_handle *h, const double *d_pos, const double *d_body_pos) {
    ProfScope ps(h, PROF_GEOMETRY);
    Geometry &g = h->geo;
    const int N = h->N;
    g.valid = false;
    ++h->geo_gen;  // captured solver graphs refer to this geometry's sizes
    CellGrid cg = make_cell_grid(h, h->d.rcut);
    PrepArgs a;
    a.N = N;
    for (int d = 0; d < 3; ++d) {
        a.L[d] = h->L[d];
        a.Ng[d] = h->d.grid[d];
        a.ntd[d] = h->ntiles_dim[d];
    }
    a.P = h->d.support;
    a.T = h->tile;
    a.cg = cg;
    if (N == 0) {
        g.valid = true;
        return CR_OK;
    }
    CR_CUDA(h, cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    prepare_kernel<<<blocks_for(N, 256), 256, 0, h->stream>>>(a, d_pos, h->m64.pos, h->m32.pos, g.wstart,
                                                               h->d_keys, g.cell_of, h->d_vals, h->d_flag);
    CR_LAUNCH(h, "prepare_kernel");
    int bad = 0;
    CR_CUDA(h, cudaMemcpyAsync(&bad, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    if (bad) return fail(h, CR_NUMERICAL, "non-finite or out-of-range bead position");
    CR_TRY(bin_beads(h, h->d_keys, h->ntiles, g.tile_count, g.tile_start, g.tile_beads));
    CR_TRY(realspace_build(h));
    if (h->user.precond != CR_PRECOND_DIAGONAL && !h->cond.ready) CR_TRY(conductor_setup(h));
    if (d_body_pos && h->B > 0) {
        CR_CUDA(h, cudaMemcpy2DAsync(h->d_bpos, sizeof(double4), d_body_pos, 3 * sizeof(double), 3 * sizeof(double),
                                     h->B, cudaMemcpyDeviceToDevice, h->stream));
    }
    g.valid = true;
    return CR_OK;
}

int neighbor_list_build(cr_handle *h, double r_list, int *d_count, int64_t *d_head, int *d_list, int64_t capacity,
                        int64_t *total) {
    if (!h->geo.valid) return fail(h, CR_NOT_READY, "positions not set");
    if (!(r_list > 0)) return fail(h, CR_BAD_PARAM, "r_list must be positive");
    for (int d = 0; d < 3; ++d)
        if (r_list > 0.5 * h->L[d]) return fail(h, CR_BAD_PARAM, "r_list above half the box");
    const int N = h->N;
    CellGrid cg = make_cell_grid(h, r_list);
    int *cell_of = nullptr, *start = nullptr, *beads = nullptr, *sorted = nullptr;
    int64_t *ends = nullptr;
    void *scratch = nullptr;
    size_t start_alloc = 0;
    int st = dalloc(h, &cell_of, (size_t)N);
    if (st == CR_OK) st = dalloc(h, &beads, (size_t)N);
    if (st == CR_OK) st = cell_bins(h, cg, cell_of, &start, &start_alloc, beads);
    int64_t cap = d_list ? capacity : 0;
    int *lst = d_list;
    if (st == CR_OK) st = build_list(h, cg, cell_of, start, beads, r_list, d_count, d_head, &lst, &cap, total, false);
    if (st == CR_OK && d_list && capacity >= *total && *total > 0) {
        if (*total > (int64_t)INT32_MAX) st = fail(h, CR_BAD_PARAM, "neighbour list too long to sort");
        if (st == CR_OK) st = dalloc(h, &ends, (size_t)N);
        if (st == CR_OK) st = dalloc(h, &sorted, (size_t)*total);
        if (st == CR_OK) {
            segment_end_kernel<<<blocks_for(N, 256), 256, 0, h->stream>>>(N, d_head, d_count, ends);
            st = check_cuda(h, cudaGetLastError(), "segment_end_kernel");
        }
        size_t bytes = 0;
        if (st == CR_OK)
            st = check_cuda(h, cub::DeviceSegmentedRadixSort::SortKeys(nullptr, bytes, d_list, sorted, (int)*total, N,
                                                                       d_head, ends, 0, 32, h->stream),
                            "SegmentedRadixSort size");
        if (st == CR_OK) st = dalloc(h, reinterpret_cast<char **>(&scratch), bytes + 256);
        if (st == CR_OK)
            st = check_cuda(h, cub::DeviceSegmentedRadixSort::SortKeys(scratch, bytes, d_list, sorted, (int)*total, N,
                                                                       d_head, ends, 0, 32, h->stream),
                            "SegmentedRadixSort");
        if (st == CR_OK)
            st = check_cuda(h, cudaMemcpyAsync(d_list, sorted, (size_t)*total * sizeof(int), cudaMemcpyDeviceToDevice,
                                               h->stream), "copy sorted list");
    }
    cudaStreamSynchronize(h->stream);
    dfree(&cell_of);
    dfree(&start);
    dfree(&beads);
    dfree(&sorted);
    dfree(&ends);
    dfree(reinterpret_cast<char **>(&scratch));
    return st;
}

}  // namespace cr
