// batch.cu -- many independent systems solved concurrently.
//
// Small systems (a few thousand charges) cannot fill a B200: one operator application
// is a chain of short kernels and every Arnoldi step waits for its Hessenberg column.
// cr_batch_compute therefore runs the systems side by side: a pool of host threads,
// each with its own non-blocking stream, takes systems largest first and runs the whole
// cr_compute on its stream, so the GPU works on up to n_threads systems at once and one
// system's host round trips hide behind the others' kernels.  Each system keeps its own
// handle and buffers, so results agree with solving the systems one by one up to the
// summation order of the atomic accumulations (spreading, real-space forces), which
// differs from run to run in either mode.
#include <algorithm>
#include <atomic>
#include <numeric>
#include <thread>
#include <vector>

#include "cr_internal.cuh"

extern "C" {

int cr_batch_compute(int n, cr_handle *const *handles, const double *const *d_pos, const double *const *d_body_pos,
                     double *const *d_q, double *const *d_phi, double *const *d_force, cr_solve_stats *stats,
                     int *status, int n_threads) {
    if (n < 0 || (n > 0 && (!handles || !d_pos || !d_body_pos || !d_q || !d_phi || !d_force || !status)))
        return CR_BAD_PARAM;
    if (n == 0) return CR_OK;
    for (int i = 0; i < n; ++i)
        if (!handles[i]) return CR_BAD_PARAM;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return CR_CUDA_ERROR;
    }
    const int T = std::max(1, std::min(n, n_threads > 0 ? n_threads : 16));
    std::vector<cudaStream_t> streams(T, nullptr);
    for (int t = 0; t < T; ++t)
        if (cudaStreamCreateWithFlags(&streams[t], cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            for (int u = 0; u < t; ++u) cudaStreamDestroy(streams[u]);
            return CR_CUDA_ERROR;
        }
    // largest systems first
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return handles[a]->N + handles[a]->B > handles[b]->N + handles[b]->B; });
    std::atomic<int> next(0);
    auto worker = [&](int t) {
        cudaSetDevice(dev);
        for (int k = next++; k < n; k = next++) {
            const int i = order[k];
            cr_handle *h = handles[i];
            cudaStream_t saved = h->stream;
            h->stream = streams[t];
            status[i] = cr_compute(h, d_pos[i], d_body_pos[i], d_q[i], d_phi[i], d_force[i], stats ? &stats[i] : nullptr);
            cudaStreamSynchronize(streams[t]);
            h->stream = saved;
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(T - 1);
    for (int t = 1; t < T; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto &th : pool) th.join();
    for (int t = 0; t < T; ++t) cudaStreamDestroy(streams[t]);
    int worst = CR_OK;
    for (int i = 0; i < n; ++i)
        if (status[i] != CR_OK && (worst == CR_OK || worst == CR_NOT_CONVERGED)) worst = status[i];
    return worst;
}

}  // extern "C"
