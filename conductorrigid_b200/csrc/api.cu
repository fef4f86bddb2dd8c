// api.cu -- the C ABI declared in include/conductor_rigid.h.
//
// The handle plays the part of the reference's ConductorRigid ForceCompute
// (ConductorRigid.h:21-112): it owns the derived parameters, tables, mesh, FFT plans,
// per-solve geometry and the Krylov workspace; the caller owns the particle arrays.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "cr_internal.cuh"

namespace cr {

int fail(cr_handle *h, int status, const std::string &msg) {
    if (h) h->last_error = msg;
    return status;
}

int check_cuda(cr_handle *h, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return CR_OK;
    cudaGetLastError();
    const int st = e == cudaErrorMemoryAllocation ? CR_OUT_OF_MEMORY : CR_CUDA_ERROR;
    return fail(h, st, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_cufft(cr_handle *h, cufftResult r, const char *what) {
    if (r == CUFFT_SUCCESS) return CR_OK;
    return fail(h, r == CUFFT_ALLOC_FAILED ? CR_OUT_OF_MEMORY : CR_CUDA_ERROR,
                std::string(what) + ": cuFFT error " + std::to_string((int)r));
}

long prof_begin(cr_handle *h, int id) {
    if (!h->prof.on) return -1;
    Profiler &p = h->prof;
    if (p.used + 2 > p.pool.size()) {
        const size_t grow = std::max<size_t>(1024, p.pool.size());
        for (size_t k = 0; k < grow; ++k) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) {
                cudaGetLastError();
                return -1;
            }
            p.pool.push_back(e);
        }
    }
    const size_t s = p.used;
    p.used += 2;
    cudaEventRecord(p.pool[s], h->stream);
    p.marks.emplace_back(id, s);
    return (long)s;
}

void prof_end(cr_handle *h, long token) {
    if (token < 0 || !h->prof.on) return;
    cudaEventRecord(h->prof.pool[(size_t)token + 1], h->stream);
}

namespace {

void free_all(cr_handle *h) {
    correction_free(h);
    conductor_free(h);
    coarse_free(h);
    mesh_free(h->m64);
    mesh_free(h->m32);
    geometry_free(h);
    krylov_free(h);
    dfree(&h->d_body);
    dfree(&h->d_rigid);
    dfree(&h->d_Q);
    dfree(&h->d_bsize);
    dfree(&h->d_body_start);
    dfree(&h->d_body_members);
    dfree(&h->d_bpos);
    dfree(&h->d_tmp_n);
    dfree(&h->d_tmp_n2);
    dfree(&h->d_force);
    dfree(&h->d_io_pos);
    dfree(&h->d_io_bpos);
    dfree(&h->d_io_q);
    dfree(&h->d_io_phi);
    dfree(&h->d_io_force);
    dfree(&h->d_bf);
    dfree(&h->d_bt);
    dfree(&h->d_moves);
    dfree(&h->d_guess);
    h->n_guess = 0;
}

int derive(cr_handle *h, const cr_params *p, const double L[3]) {
    cr_derived d;
    const int st = cr_derive_params(p, L, &d);
    if (st == CR_GRID_TOO_LARGE) return fail(h, st, "requested number of Fourier nodes exceeds maximum of 4096");
    if (st != CR_OK) return fail(h, st, "invalid parameters (xi, errortol, box, or rcut above half the box)");
    h->user = *p;
    h->d = d;
    for (int k = 0; k < 3; ++k) {
        h->L[k] = L[k];
        h->field[k] = p->field[k];
    }
    const int nt = d.n_table + 1;
    h->h_phiq.assign(2 * (size_t)nt, 0.0);
    h->h_gradphiq.assign(2 * (size_t)nt, 0.0);
    cr_build_tables(&d, p->xi, h->h_phiq.data(), h->h_gradphiq.data());
    // tiles of 8^3 nodes (fewer along short dimensions); cr_autotune may change this
    h->tile = 8;
    h->spread_mode = 0;
    h->ntiles = 1;
    for (int k = 0; k < 3; ++k) {
        h->ntiles_dim[k] = (d.grid[k] + h->tile - 1) / h->tile;
        h->ntiles *= h->ntiles_dim[k];
    }
    return CR_OK;
}

// Allocate every device structure for the current parameters and topology size.
int realize(cr_handle *h) {
    CR_TRY(mesh_init(h, h->m64));
    CR_TRY(mesh_init(h, h->m32));
    CR_TRY(geometry_alloc(h));
    CR_TRY(krylov_alloc(h));
    CR_TRY(dalloc(h, &h->d_bpos, (size_t)std::max(h->B, 1)));
    CR_TRY(dalloc(h, &h->d_tmp_n, (size_t)(h->N + h->B)));
    CR_TRY(dalloc(h, &h->d_tmp_n2, (size_t)(h->N + h->B)));
    CR_TRY(dalloc(h, &h->d_force, 3 * (size_t)h->N));
    CR_CUDA(h, cudaMemset(h->d_bpos, 0, sizeof(double4) * std::max(h->B, 1)));
    return CR_OK;
}

int need_ready(cr_handle *h) {
    if (!h) return CR_BAD_PARAM;
    if (!h->have_topology) return fail(h, CR_NOT_READY, "topology not set");
    return CR_OK;
}

int need_geometry(cr_handle *h) {
    CR_TRY(need_ready(h));
    if (!h->geo.valid) return fail(h, CR_NOT_READY, "positions not set");
    return CR_OK;
}

bool finite_params(const cr_params *p) {
    if (p->precond != CR_PRECOND_DIAGONAL && p->precond != CR_PRECOND_CONDUCTOR &&
        p->precond != CR_PRECOND_TWO_LEVEL)
        return false;
    if (p->precision < CR_FP64 || p->precision > CR_FP32) return false;
    if (!std::isfinite(p->xi) || !std::isfinite(p->errortol) || !std::isfinite(p->rcut) ||
        !std::isfinite(p->gmres_tol))
        return false;
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(p->field[k])) return false;
    return true;
}

template <typename R> int wave_out(cr_handle *h, MeshBuffers<R> &m, const double *d_q, double *d_phi) {
    CR_TRY(cast_charges(h, m, d_q));
    CR_TRY(wave_potential(h, m));
    CR_TRY(cast_to_double(h, m.phi, d_phi, h->N));
    return CR_OK;
}

}  // namespace
}  // namespace cr

using namespace cr;

namespace cr {
// out += sum_i a_i b_i / 2 (FP64; one atomic per block)
__global__ void half_dot_kernel(int n, const double *__restrict__ a, const double *__restrict__ b, double *out) {
    __shared__ double red[8];
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * b[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicAdd(out, 0.5 * t);
    }
}
}  // namespace cr

extern "C" {

int cr_abi_version(void) { return CR_ABI_VERSION; }

const char *cr_status_string(int s) {
    switch (s) {
        case CR_OK: return "ok";
        case CR_NOT_CONVERGED: return "not converged";
        case CR_BAD_PARAM: return "bad parameter";
        case CR_CUDA_ERROR: return "CUDA error";
        case CR_TIMEOUT: return "timeout";
        case CR_OUT_OF_MEMORY: return "out of memory";
        case CR_GRID_TOO_LARGE: return "grid too large";
        case CR_NOT_READY: return "not ready";
        case CR_NUMERICAL: return "non-finite value";
        default: return "unknown status";
    }
}

const char *cr_last_error(const cr_handle *h) { return h ? h->last_error.c_str() : "null handle"; }

int cr_create(const cr_params *p, const double L[3], cr_handle **out) {
    if (!p || !L || !out) return CR_BAD_PARAM;
    *out = nullptr;
    if (!finite_params(p)) return CR_BAD_PARAM;
    cr_handle *h = new cr_handle();
    const int st = derive(h, p, L);
    if (st != CR_OK) {
        delete h;
        return st;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        return CR_CUDA_ERROR;
    }
    if (cudaDeviceGetAttribute(&h->n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || h->n_sm <= 0) {
        cudaGetLastError();
        delete h;
        return CR_CUDA_ERROR;
    }
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    *out = h;
    return CR_OK;
}

int cr_destroy(cr_handle *h) {
    if (!h) return CR_BAD_PARAM;
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    free_all(h);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    for (cudaEvent_t e : h->prof.pool) cudaEventDestroy(e);
    delete h;
    return CR_OK;
}

int cr_get_derived(const cr_handle *h, cr_derived *out) {
    if (!h || !out) return CR_BAD_PARAM;
    *out = h->d;
    return CR_OK;
}

int cr_set_field(cr_handle *h, const double field[3]) {
    if (!h || !field) return CR_BAD_PARAM;
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(field[k])) return fail(h, CR_BAD_PARAM, "non-finite field");
    for (int k = 0; k < 3; ++k) {
        h->field[k] = field[k];
        h->user.field[k] = field[k];
    }
    return CR_OK;
}

int cr_set_params(cr_handle *h, const cr_params *p, const double L[3]) {
    if (!h || !p || !L) return CR_BAD_PARAM;
    if (!finite_params(p)) return fail(h, CR_BAD_PARAM, "non-finite parameter");
    if (h->stream) cudaStreamSynchronize(h->stream);
    CR_TRY(derive(h, p, L));
    h->geo.valid = false;
    if (h->have_topology) {
        conductor_free(h);
        coarse_free(h);
        mesh_free(h->m64);
        mesh_free(h->m32);
        geometry_free(h);
        krylov_free(h);
        CR_TRY(realize(h));
    }
    return CR_OK;
}

int cr_set_stream(cr_handle *h, void *stream) {
    if (!h) return CR_BAD_PARAM;
    h->stream = (cudaStream_t)stream;
    return CR_OK;
}

int cr_set_tiling(cr_handle *h, int tile_edge, int spread_mode) {
    CR_TRY(need_ready(h));
    if (spread_mode < 0 || spread_mode > 1) return fail(h, CR_BAD_PARAM, "spread mode must be 0 or 1");
    if (h->stream) CR_CUDA(h, cudaStreamSynchronize(h->stream));
    CR_TRY(mesh_set_tile(h, tile_edge));
    h->spread_mode = spread_mode;
    return CR_OK;
}

// Time the FP32 mesh path (spread, FFT, influence function, FFT, contract) of the given
// positions for every valid tiling and keep the fastest.
int cr_autotune(cr_handle *h, const double *d_pos, const double *d_body_pos, int reps, int *tile_edge,
                int *spread_mode, float *best_ms) {
    CR_TRY(need_ready(h));
    if (h->N > 0 && !d_pos) return fail(h, CR_BAD_PARAM, "null positions");
    if (h->B > 0 && !d_body_pos) return fail(h, CR_BAD_PARAM, "null body positions");
    reps = std::max(1, reps);
    const bool compiled = h->d.support == 9 || h->d.support == 11;
    const int edges[] = {4, 6, 8, 12, 16};
    int best_t = h->tile, best_m = h->spread_mode;
    float best = 3.4e38f;
    if (h->N > 0) {
        for (int t : edges) {
            for (int mode = 0; mode < 2; ++mode) {
                if (mode == 0 && !(t == 8 && compiled)) continue;  // register columns exist for T = 8 only
                if (mesh_set_tile(h, t) != CR_OK) continue;             // too large for shared memory
                h->spread_mode = mode;
                CR_TRY(geometry_update(h, d_pos, d_body_pos));
                CR_TRY(cast_charges(h, h->m32, d_pos));                 // any charges will do for timing
                CR_TRY(wave_potential(h, h->m32));
                CR_CUDA(h, cudaEventRecord(h->ev0, h->stream));
                for (int r = 0; r < reps; ++r) CR_TRY(wave_potential(h, h->m32));
                CR_CUDA(h, cudaEventRecord(h->ev1, h->stream));
                CR_CUDA(h, cudaEventSynchronize(h->ev1));
                float ms = 0.f;
                CR_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
                ms /= reps;
                if (ms < best) {
                    best = ms;
                    best_t = t;
                    best_m = mode;
                }
            }
        }
    }
    CR_TRY(mesh_set_tile(h, best_t));
    h->spread_mode = best_m;
    CR_TRY(geometry_update(h, d_pos, d_body_pos));
    if (tile_edge) *tile_edge = best_t;
    if (spread_mode) *spread_mode = best_m;
    if (best_ms) *best_ms = h->N > 0 ? best : 0.f;
    return CR_OK;
}

int cr_set_graphs(cr_handle *h, int enable) {
    if (!h) return CR_BAD_PARAM;
    h->use_graphs = enable ? 1 : 0;
    return CR_OK;
}

int cr_set_correction(cr_handle *h, cr_mlp *net, double weight) {
    if (!h) return CR_BAD_PARAM;
    if (!std::isfinite(weight)) return fail(h, CR_BAD_PARAM, "non-finite correction weight");
    if (h->stream) CR_CUDA(h, cudaStreamSynchronize(h->stream));
    h->corr.net = net;
    h->corr.weight = weight;
    h->corr.active = 0;
    return CR_OK;
}

int cr_correction_samples(cr_handle *h, int max_dirs, uint16_t *d_x, float *d_t, int *rows) {
    if (!h || !rows || max_dirs < 0) return CR_BAD_PARAM;
    *rows = 0;
    if (!h->corr.net) return fail(h, CR_NOT_READY, "no correction network set");
    if (!h->geo.valid) return fail(h, CR_NOT_READY, "no solve on this handle yet");
    if (max_dirs > 0 && (!d_x || !d_t)) return fail(h, CR_BAD_PARAM, "null output");
    if ((uintptr_t)d_x % 16) return fail(h, CR_BAD_PARAM, "feature rows must be 16-byte aligned");
    return correction_samples(h, max_dirs, d_x, d_t, rows);
}

int cr_set_realspace(cr_handle *h, int flags) {
    if (!h) return CR_BAD_PARAM;
    if (flags & ~(CR_REALSPACE_ONFLY32 | CR_REALSPACE_ONFLY64 | CR_REALSPACE_STREAM | CR_REALSPACE_SERIAL))
        return fail(h, CR_BAD_PARAM, "unknown real-space flags");
    if (h->stream) CR_CUDA(h, cudaStreamSynchronize(h->stream));
    h->rs_onfly = flags;
    h->geo_gen++;  // captured Arnoldi steps hold the old kernels: capture again
    return CR_OK;
}

int cr_set_wait_limit(cr_handle *h, long long cycles, int withhold_next) {
    if (!h) return CR_BAD_PARAM;
    if (h->stream) CR_CUDA(h, cudaStreamSynchronize(h->stream));
    h->rs.wait_limit = cycles > 0 ? cycles : (1LL << 31);
    h->rs.withhold_next = withhold_next ? 1 : 0;
    h->geo_gen++;  // captured Arnoldi steps hold the old limit: capture again
    return CR_OK;
}

int cr_graph_launches(const cr_handle *h, long long *launches) {
    if (!h || !launches) return CR_BAD_PARAM;
    *launches = h->graph_launches;
    return CR_OK;
}

int cr_set_topology(cr_handle *h, int n_beads, const uint32_t *body, int n_bodies, const uint8_t *rigid,
                    const double *body_charge) {
    if (!h || n_beads < 0 || n_bodies < 0) return CR_BAD_PARAM;
    if (n_beads > 0 && (!body || n_bodies == 0)) return fail(h, CR_BAD_PARAM, "missing body list");
    if (n_bodies > 0 && (!rigid || !body_charge)) return fail(h, CR_BAD_PARAM, "missing body arrays");
    std::vector<int> size(n_bodies, 0);
    for (int i = 0; i < n_beads; ++i) {
        if (body[i] >= (uint32_t)n_bodies) return fail(h, CR_BAD_PARAM, "body tag out of range");
        size[body[i]]++;
    }
    for (int b = 0; b < n_bodies; ++b) {
        if (size[b] == 0) return fail(h, CR_BAD_PARAM, "body without beads");
        if (!rigid[b] && size[b] != 1) return fail(h, CR_BAD_PARAM, "a free bead body must hold exactly one bead");
        if (!std::isfinite(body_charge[b])) return fail(h, CR_BAD_PARAM, "non-finite body charge");
    }
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    h->have_topology = false;
    h->N = n_beads;
    h->B = n_bodies;
    // host member lists: beads of each body in ascending bead index
    h->h_body_start.assign((size_t)n_bodies + 1, 0);
    for (int b = 0; b < n_bodies; ++b) h->h_body_start[b + 1] = h->h_body_start[b] + size[b];
    h->h_body_members.assign((size_t)n_beads, 0);
    {
        std::vector<int> fill(h->h_body_start.begin(), h->h_body_start.end() - 1);
        for (int i = 0; i < n_beads; ++i) h->h_body_members[fill[body[i]]++] = i;
    }
    CR_TRY(dalloc(h, &h->d_body, (size_t)std::max(n_beads, 1)));
    CR_TRY(dalloc(h, &h->d_rigid, (size_t)std::max(n_bodies, 1)));
    CR_TRY(dalloc(h, &h->d_Q, (size_t)std::max(n_bodies, 1)));
    CR_TRY(dalloc(h, &h->d_bsize, (size_t)std::max(n_bodies, 1)));
    CR_TRY(dalloc(h, &h->d_body_start, (size_t)n_bodies + 1));
    CR_TRY(dalloc(h, &h->d_body_members, (size_t)std::max(n_beads, 1)));
    if (n_beads) CR_CUDA(h, cudaMemcpy(h->d_body, body, n_beads * sizeof(uint32_t), cudaMemcpyHostToDevice));
    if (n_bodies) {
        CR_CUDA(h, cudaMemcpy(h->d_rigid, rigid, n_bodies, cudaMemcpyHostToDevice));
        CR_CUDA(h, cudaMemcpy(h->d_Q, body_charge, n_bodies * sizeof(double), cudaMemcpyHostToDevice));
    }
    CR_TRY(realize(h));
    if (n_beads) CR_TRY(topology_build(h));
    h->have_topology = true;
    return CR_OK;
}

int cr_set_positions(cr_handle *h, const double *d_pos, const double *d_body_pos) {
    CR_TRY(need_ready(h));
    if (!d_pos && h->N > 0) return fail(h, CR_BAD_PARAM, "null positions");
    CR_TRY(geometry_update(h, d_pos, d_body_pos));
    return CR_OK;
}

int cr_apply_operator(cr_handle *h, const double *d_x, double *d_y, int precision) {
    CR_TRY(need_geometry(h));
    if (h->N == 0) return CR_OK;
    if (!d_x || !d_y) return fail(h, CR_BAD_PARAM, "null vector");
    CR_TRY(apply_operator(h, d_x, d_y, precision));
    CR_TRY(check_cuda(h, cudaStreamSynchronize(h->stream), "cr_apply_operator"));
    return realspace_check(h);
}

int cr_precondition(cr_handle *h, const double *d_x, double *d_y) {
    CR_TRY(need_ready(h));
    if (h->N == 0) return CR_OK;
    if (!d_x || !d_y) return fail(h, CR_BAD_PARAM, "null vector");
    CR_TRY(coarse_prepare(h));
    CR_TRY(precondition(h, d_x, d_y));
    return check_cuda(h, cudaStreamSynchronize(h->stream), "cr_precondition");
}

int cr_coarse_info(cr_handle *h, int *active, int *n_coarse, long long *n_pairs, int *n_modes, int *sparse) {
    CR_TRY(need_ready(h));
    CR_TRY(coarse_prepare(h));
    const CoarseSpace &c = h->coarse;
    const bool on = h->user.precond == CR_PRECOND_TWO_LEVEL && c.active;
    if (active) *active = on ? 1 : 0;
    if (n_coarse) *n_coarse = on ? c.nc : 0;
    if (n_pairs) *n_pairs = on ? c.npairs : 0;
    if (n_modes) *n_modes = on ? c.nmodes : 0;
    if (sparse) *sparse = on && c.sparse ? 1 : 0;
    return check_cuda(h, cudaStreamSynchronize(h->stream), "cr_coarse_info");
}

int cr_set_coarse(cr_handle *h, int max_dense, int pcg_iterations) {
    if (!h) return CR_BAD_PARAM;
    if (max_dense < 0 || pcg_iterations < 0 || pcg_iterations > 64)
        return fail(h, CR_BAD_PARAM, "cr_set_coarse: max_dense >= 0 and 0 <= pcg_iterations <= 64");
    h->coarse.max_dense = max_dense;
    h->coarse.pcg_iters = pcg_iterations;
    h->coarse.gen = -1;                                // rebuilt by the next solve
    h->kry.exec_gen[0] = h->kry.exec_gen[1] = -1;      // captured steps hold the old sequence
    return CR_OK;
}

int cr_objective(cr_handle *h, double *d_rhs) {
    CR_TRY(need_geometry(h));
    if (h->N == 0) return CR_OK;
    if (!d_rhs) return fail(h, CR_BAD_PARAM, "null vector");
    CR_TRY(objective(h, d_rhs));
    return check_cuda(h, cudaStreamSynchronize(h->stream), "cr_objective");
}

int cr_wave_potential(cr_handle *h, const double *d_q, double *d_phi, int precision) {
    CR_TRY(need_geometry(h));
    if (h->N == 0) return CR_OK;
    if (!d_q || !d_phi) return fail(h, CR_BAD_PARAM, "null vector");
    if (precision == CR_FP64) CR_TRY(wave_out(h, h->m64, d_q, d_phi));
    else CR_TRY(wave_out(h, h->m32, d_q, d_phi));
    return check_cuda(h, cudaStreamSynchronize(h->stream), "cr_wave_potential");
}

int cr_spread(cr_handle *h, const double *d_q, double *d_grid, int precision) {
    CR_TRY(need_geometry(h));
    if (!d_grid) return fail(h, CR_BAD_PARAM, "null vector");
    const long G = grid_size(h);
    if (h->N == 0) return check_cuda(h, cudaMemset(d_grid, 0, G * sizeof(double)), "cr_spread");
    if (!d_q) return fail(h, CR_BAD_PARAM, "null vector");
    if (precision == CR_FP64) {
        CR_TRY(cast_charges(h, h->m64, d_q));
        CR_TRY(spread_only(h, h->m64));
        CR_CUDA(h, cudaMemcpyAsync(d_grid, h->m64.grid, G * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    } else {
        CR_TRY(cast_charges(h, h->m32, d_q));
        CR_TRY(spread_only(h, h->m32));
        CR_TRY(cast_to_double(h, h->m32.grid, d_grid, G));
    }
    return check_cuda(h, cudaStreamSynchronize(h->stream), "cr_spread");
}


// Electrostatic energy of the bead charges, U = 1/2 q.(M q), with M the periodic
// (Ewald-split) shell interaction of the current positions, FP64.
int cr_energy(cr_handle *h, const double *d_q, double *energy) {
    CR_TRY(need_geometry(h));
    if (!energy) return fail(h, CR_BAD_PARAM, "null output");
    *energy = 0.0;
    if (h->N == 0) return CR_OK;
    if (!d_q) return fail(h, CR_BAD_PARAM, "null vector");
    CR_TRY(cr_apply_M(h, d_q, h->d_tmp_n, CR_FP64));
    CR_CUDA(h, cudaMemsetAsync(h->d_tmp_n2, 0, sizeof(double), h->stream));
    cr::half_dot_kernel<<<std::min(4 * 148, blocks_for(h->N, 256)), 256, 0, h->stream>>>(h->N, d_q, h->d_tmp_n,
                                                                                     h->d_tmp_n2);
    CR_LAUNCH(h, "half_dot_kernel");
    CR_CUDA(h, cudaMemcpyAsync(energy, h->d_tmp_n2, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    return check_cuda(h, cudaStreamSynchronize(h->stream), "cr_energy");
}

int cr_virial(cr_handle *h, const double *d_q, double *virial) {
    CR_TRY(need_geometry(h));
    if (!virial) return fail(h, CR_BAD_PARAM, "null output");
    for (int e = 0; e < 13; ++e) virial[e] = 0.0;
    if (h->N == 0) return CR_OK;
    if (!d_q) return fail(h, CR_BAD_PARAM, "null vector");
    CR_TRY(cast_charges(h, h->m64, d_q));
    CR_TRY(real_space_virial(h, d_q, virial));
    return wave_virial(h, virial + 6);
}

int cr_apply_M(cr_handle *h, const double *d_q, double *d_Mq, int precision) {
    CR_TRY(need_geometry(h));
    if (h->N == 0) return CR_OK;
    if (!d_q || !d_Mq) return fail(h, CR_BAD_PARAM, "null vector");
    if (precision == CR_FP64) {
        CR_TRY(cast_charges(h, h->m64, d_q));
        CR_TRY(wave_potential(h, h->m64));
        CR_TRY(real_space_apply(h, h->m64, nullptr, d_Mq));
    } else {
        CR_TRY(cast_charges(h, h->m32, d_q));
        CR_TRY(wave_potential(h, h->m32));
        CR_TRY(real_space_apply(h, h->m32, nullptr, d_Mq));
    }
    return check_cuda(h, cudaStreamSynchronize(h->stream), "cr_apply_M");
}

int cr_forces(cr_handle *h, const double *d_q, double *d_force, int precision) {
    CR_TRY(need_geometry(h));
    if (h->N == 0) return CR_OK;
    if (!d_q || !d_force) return fail(h, CR_BAD_PARAM, "null vector");
    if (precision == CR_FP64) {
        CR_TRY(cast_charges(h, h->m64, d_q));
        CR_TRY(wave_force(h, h->m64));
        CR_TRY(real_space_force(h, h->m64, d_q, d_force));
    } else {
        CR_TRY(cast_charges(h, h->m32, d_q));
        CR_TRY(wave_force(h, h->m32));
        CR_TRY(real_space_force(h, h->m32, d_q, d_force));
    }
    return check_cuda(h, cudaStreamSynchronize(h->stream), "cr_forces");
}

int cr_profile(cr_handle *h, int enable) {
    if (!h) return CR_BAD_PARAM;
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    h->prof.on = enable != 0;
    h->prof.used = 0;
    h->prof.marks.clear();
    return CR_OK;
}

int cr_profile_read(cr_handle *h, int kernel_class, int *launches, double *total_ms) {
    if (!h || !launches || !total_ms || kernel_class < 0 || kernel_class >= PROF_COUNT) return CR_BAD_PARAM;
    CR_CUDA(h, h->stream ? cudaStreamSynchronize(h->stream) : cudaDeviceSynchronize());
    int n = 0;
    double t = 0.0;
    for (const auto &m : h->prof.marks) {
        if (m.first != kernel_class) continue;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, h->prof.pool[m.second], h->prof.pool[m.second + 1]) == cudaSuccess) {
            ++n;
            t += ms;
        } else {
            cudaGetLastError();
        }
    }
    *launches = n;
    *total_ms = t;
    return CR_OK;
}

int cr_get_geometry_info(const cr_handle *h, cr_geometry_info *out) {
    if (!h || !out) return CR_BAD_PARAM;
    out->real_space_pairs = h->geo.valid ? h->geo.nl_total : 0;
    out->tile_edge = h->tile;
    out->n_tiles = h->ntiles;
    out->n_beads = h->N;
    out->n_bodies = h->B;
    out->cluster_pairs = h->geo.valid ? h->rs.npairs : 0;
    out->stored_values = h->geo.valid ? h->rs.nnz : 0;
    return CR_OK;
}

int cr_counters(const cr_handle *h, long long *kernel_launches, long long *fft_execs) {
    if (!h || !kernel_launches || !fft_execs) return CR_BAD_PARAM;
    *kernel_launches = h->launches;
    *fft_execs = h->fft_execs;
    return CR_OK;
}

int cr_neighbor_list(cr_handle *h, double r_list, int *d_count, int64_t *d_head, int *d_list, int64_t capacity,
                     int64_t *total) {
    CR_TRY(need_geometry(h));
    if (!total || capacity < 0) return fail(h, CR_BAD_PARAM, "null output");
    if (h->N == 0) {
        *total = 0;
        return CR_OK;
    }
    if (!d_count || !d_head) return fail(h, CR_BAD_PARAM, "null output");
    return neighbor_list_build(h, r_list, d_count, d_head, capacity > 0 ? d_list : nullptr, capacity, total);
}

// gpu_ComputeForce (ConductorRigid.cu:1153-1286): geometry, right-hand side, solve
// from the warm start, write back charges and potentials, then the force pass.
int cr_compute(cr_handle *h, const double *d_pos, const double *d_body_pos, double *d_q, double *d_phi,
               double *d_force, cr_solve_stats *stats) {
    CR_TRY(need_ready(h));
    if ((!d_pos || !d_q || !d_force) && h->N > 0) return fail(h, CR_BAD_PARAM, "null array");
    if ((!d_phi || !d_body_pos) && h->B > 0) return fail(h, CR_BAD_PARAM, "null body array");
    const int N = h->N, B = h->B;
    cr_solve_stats st{};
    if (N == 0) {
        st.converged = 1;
        if (stats) *stats = st;
        return CR_OK;
    }
    CR_TRY(geometry_update(h, d_pos, d_body_pos));
    Krylov &K = h->kry;
    CR_TRY(objective(h, K.b));
    CR_CUDA(h, cudaMemcpyAsync(K.x, d_q, N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (B) CR_CUDA(h, cudaMemcpyAsync(K.x + N, d_phi, B * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CR_CUDA(h, cudaEventRecord(h->ev0, h->stream));
    const int sst = solve(h, K.x, K.b, &st);
    if (sst != CR_OK && sst != CR_NOT_CONVERGED) {
        const int rc = realspace_check(h);  // a wait that ran out explains a failed solve
        return rc != CR_OK ? rc : sst;
    }
    CR_CUDA(h, cudaEventRecord(h->ev1, h->stream));
    CR_CUDA(h, cudaMemcpyAsync(d_q, K.x, N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (B) CR_CUDA(h, cudaMemcpyAsync(d_phi, K.x + N, B * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    // force pass in FP64
    CR_TRY(cast_charges(h, h->m64, K.x));
    CR_TRY(wave_force(h, h->m64));
    CR_TRY(real_space_force(h, h->m64, K.x, d_force));
    CR_CUDA(h, cudaStreamSynchronize(h->stream));
    CR_TRY(realspace_check(h));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    st.solve_ms = ms;
    if (stats) *stats = st;
    if (sst == CR_NOT_CONVERGED) fail(h, CR_NOT_CONVERGED, "GMRES reached its iteration limit");
    return sst;
}

int cr_compute_host(cr_handle *h, const double *pos, const double *body_pos, double *q, double *phi, double *force,
                    cr_solve_stats *stats) {
    CR_TRY(need_ready(h));
    const int N = h->N, B = h->B;
    if ((!pos || !q || !force) && N > 0) return fail(h, CR_BAD_PARAM, "null array");
    if ((!phi || !body_pos) && B > 0) return fail(h, CR_BAD_PARAM, "null body array");
    if (!h->d_io_pos) {
        CR_TRY(dalloc(h, &h->d_io_pos, 3 * (size_t)std::max(N, 1)));
        CR_TRY(dalloc(h, &h->d_io_bpos, 3 * (size_t)std::max(B, 1)));
        CR_TRY(dalloc(h, &h->d_io_q, (size_t)std::max(N, 1)));
        CR_TRY(dalloc(h, &h->d_io_phi, (size_t)std::max(B, 1)));
        CR_TRY(dalloc(h, &h->d_io_force, 3 * (size_t)std::max(N, 1)));
    }
    cudaStream_t s = h->stream;
    CR_CUDA(h, cudaMemcpyAsync(h->d_io_pos, pos, 3 * (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s));
    CR_CUDA(h, cudaMemcpyAsync(h->d_io_q, q, (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s));
    if (B) {
        CR_CUDA(h, cudaMemcpyAsync(h->d_io_bpos, body_pos, 3 * (size_t)B * sizeof(double), cudaMemcpyHostToDevice, s));
        CR_CUDA(h, cudaMemcpyAsync(h->d_io_phi, phi, (size_t)B * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    const int st = cr_compute(h, h->d_io_pos, h->d_io_bpos, h->d_io_q, h->d_io_phi, h->d_io_force, stats);
    if (st != CR_OK && st != CR_NOT_CONVERGED) return st;
    CR_CUDA(h, cudaMemcpyAsync(q, h->d_io_q, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (B) CR_CUDA(h, cudaMemcpyAsync(phi, h->d_io_phi, (size_t)B * sizeof(double), cudaMemcpyDeviceToHost, s));
    CR_CUDA(h, cudaMemcpyAsync(force, h->d_io_force, 3 * (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, s));
    CR_CUDA(h, cudaStreamSynchronize(s));
    return st;
}

int cr_body_force_torque(cr_handle *h, const double *d_pos, const double *d_body_pos, const double *d_force,
                         double *d_body_force, double *d_body_torque) {
    CR_TRY(need_ready(h));
    if (h->B > 0 && (!d_pos || !d_body_pos || !d_force || !d_body_force || !d_body_torque))
        return fail(h, CR_BAD_PARAM, "null array");
    return body_force_torque(h, d_pos, d_body_pos, d_force, d_body_force, d_body_torque);
}

int cr_brownian_step(cr_handle *h, const cr_brownian_params *p, int64_t step, const double *d_radius,
                     const double *d_force, double *d_pos, double *d_body_pos) {
    CR_TRY(need_ready(h));
    if (!p) return fail(h, CR_BAD_PARAM, "null parameters");
    if (!(p->dt >= 0.0) || !(p->kT >= 0.0) || !(p->viscosity > 0.0) || !std::isfinite(p->dt) ||
        !std::isfinite(p->kT) || !std::isfinite(p->viscosity))
        return fail(h, CR_BAD_PARAM, "dt and kT must be finite and >= 0, viscosity > 0");
    if (!(p->repulsion >= 0.0) || !std::isfinite(p->repulsion) || !std::isfinite(p->contact_gap))
        return fail(h, CR_BAD_PARAM, "repulsion must be finite and >= 0");
    if (h->B > 0 && (!d_radius || !d_force || !d_pos || !d_body_pos)) return fail(h, CR_BAD_PARAM, "null array");
    const int st = brownian_step(h, p, (long long)step, d_radius, d_force, d_pos, d_body_pos);
    h->geo.valid = false;  // positions moved: the next solve rebuilds the geometry
    return st;
}

}  // extern "C"
