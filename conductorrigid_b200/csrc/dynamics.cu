// dynamics.cu -- bead-to-body force/torque reduction and an overdamped rigid-body
// Brownian step.
//
// The reference leaves time integration to HOOMD's rigid-body integrator, which this
// library does not have; the dynamics workload needs one.  Per body (one warp):
//   F_b = sum F_i,  tau_b = sum (r_i - R_b) x F_i            (minimum image, FP64)
//   dR  = mu_t F_b dt + sqrt(2 kT mu_t dt) xi_t,   mu_t = 1/(6 pi eta a_b)
//   dth = mu_r tau_b dt + sqrt(2 kT mu_r dt) xi_r, mu_r = 1/(8 pi eta a_b^3)
//   R_b <- R_b + dR,  r_i <- R_b + dR + Rot(dth) (r_i - R_b)   (Rodrigues rotation)
// and every position is wrapped back into the box.  Free beads (rigid = 0) translate
// only.  An optional harmonic steric repulsion between body surfaces is added to F_b
// (the reference's users run one in HOOMD beside the plugin).  The Gaussian numbers come from a counter-based generator (SplitMix64 of seed,
// step, body, component; Box-Muller), so a step is reproducible anywhere.
#include <cmath>

#include "cr_internal.cuh"

namespace cr {

namespace {

__host__ __device__ inline unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform in (0, 1] from (seed, step, body, k).
__device__ inline double unit_uniform(unsigned long long seed, long long step, int body, int k) {
    unsigned long long z = mix64(seed ^ mix64((unsigned long long)step * 0x100000001B3ull + 0x51ull));
    z = mix64(z ^ ((unsigned long long)(unsigned)body << 8) ^ (unsigned long long)k);
    return ((double)(z >> 11) + 1.0) * (1.0 / 9007199254740992.0);
}

// Six standard normals for body b (Box-Muller on three uniform pairs).
__device__ inline void normals6(unsigned long long seed, long long step, int body, double *g) {
    for (int k = 0; k < 3; ++k) {
        const double u1 = unit_uniform(seed, step, body, 2 * k);
        const double u2 = unit_uniform(seed, step, body, 2 * k + 1);
        const double r = sqrt(-2.0 * log(u1));
        g[2 * k] = r * cos(2.0 * kPi * u2);
        g[2 * k + 1] = r * sin(2.0 * kPi * u2);
    }
}

__device__ inline double mimg(double d, double L) { return d - L * rint(d / L); }
__device__ inline double wrapc(double x, double L) { return x - L * floor((x + 0.5 * L) / L); }

__global__ void body_force_torque_kernel(int B, const int *__restrict__ start, const int *__restrict__ members,
                                         const double *__restrict__ pos, const double *__restrict__ bpos,
                                         const double *__restrict__ force, double Lx, double Ly, double Lz,
                                         double *__restrict__ bf, double *__restrict__ bt) {
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= B) return;
    double f[3] = {0, 0, 0}, t[3] = {0, 0, 0};
    const double c[3] = {bpos[3 * (size_t)b], bpos[3 * (size_t)b + 1], bpos[3 * (size_t)b + 2]};
    for (int k = start[b] + lane; k < start[b + 1]; k += 32) {
        const int i = members[k];
        const double r[3] = {mimg(pos[3 * (size_t)i] - c[0], Lx), mimg(pos[3 * (size_t)i + 1] - c[1], Ly),
                             mimg(pos[3 * (size_t)i + 2] - c[2], Lz)};
        const double F[3] = {force[3 * (size_t)i], force[3 * (size_t)i + 1], force[3 * (size_t)i + 2]};
        for (int d = 0; d < 3; ++d) f[d] += F[d];
        t[0] += r[1] * F[2] - r[2] * F[1];
        t[1] += r[2] * F[0] - r[0] * F[2];
        t[2] += r[0] * F[1] - r[1] * F[0];
    }
    for (int d = 0; d < 3; ++d)
        for (int o = 16; o > 0; o >>= 1) {
            f[d] += __shfl_xor_sync(0xffffffffu, f[d], o);
            t[d] += __shfl_xor_sync(0xffffffffu, t[d], o);
        }
    if (lane == 0)
        for (int d = 0; d < 3; ++d) {
            bf[3 * (size_t)b + d] = f[d];
            bt[3 * (size_t)b + d] = t[d];
        }
}

// Harmonic steric repulsion between body surfaces, added to bf: all pairs, minimum
// image, centres staged through shared memory in tiles.
__global__ void repulsion_kernel(int B, const double *__restrict__ bpos, const double *__restrict__ radius,
                                 double k, double gap, double Lx, double Ly, double Lz, double *__restrict__ bf) {
    __shared__ double4 tile[256];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    double4 c = make_double4(0, 0, 0, 0);
    if (b < B) c = make_double4(bpos[3 * (size_t)b], bpos[3 * (size_t)b + 1], bpos[3 * (size_t)b + 2], radius[b]);
    double f[3] = {0, 0, 0};
    for (int t0 = 0; t0 < B; t0 += 256) {
        const int j = t0 + threadIdx.x;
        if (j < B) tile[threadIdx.x] = make_double4(bpos[3 * (size_t)j], bpos[3 * (size_t)j + 1], bpos[3 * (size_t)j + 2], radius[j]);
        __syncthreads();
        const int cnt = min(256, B - t0);
        if (b < B)
            for (int u = 0; u < cnt; ++u) {
                if (t0 + u == b) continue;
                const double dx = mimg(tile[u].x - c.x, Lx), dy = mimg(tile[u].y - c.y, Ly), dz = mimg(tile[u].z - c.z, Lz);
                const double reach = c.w + tile[u].w + gap;
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 >= reach * reach || d2 == 0.0) continue;
                const double d = sqrt(d2);
                const double mag = k * (reach - d) / d;
                f[0] -= mag * dx;
                f[1] -= mag * dy;
                f[2] -= mag * dz;
            }
        __syncthreads();
    }
    if (b < B)
        for (int e = 0; e < 3; ++e) bf[3 * (size_t)b + e] += f[e];
}

struct StepArgs {
    double dt, kT, eta;
    unsigned long long seed;
    long long step;
    double L[3];
};

__global__ void brownian_kernel(int B, StepArgs a, const int *__restrict__ start, const int *__restrict__ members,
                                const uint8_t *__restrict__ rigid, const double *__restrict__ radius,
                                const double *__restrict__ bf, const double *__restrict__ bt,
                                double *__restrict__ pos, double *__restrict__ bpos, double *__restrict__ moves) {
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= B) return;
    const double rad = radius[b];
    const double mt = 1.0 / (6.0 * kPi * a.eta * rad);
    const double mr = 1.0 / (8.0 * kPi * a.eta * rad * rad * rad);
    double g[6];
    normals6(a.seed, a.step, b, g);
    const double st = sqrt(2.0 * a.kT * mt * a.dt), sr = sqrt(2.0 * a.kT * mr * a.dt);
    double dR[3], th[3];
    for (int d = 0; d < 3; ++d) {
        dR[d] = mt * bf[3 * (size_t)b + d] * a.dt + st * g[d];
        th[d] = rigid[b] ? mr * bt[3 * (size_t)b + d] * a.dt + sr * g[3 + d] : 0.0;
    }
    // Rodrigues rotation matrix of the angle vector th
    const double ang = sqrt(th[0] * th[0] + th[1] * th[1] + th[2] * th[2]);
    double Rm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (ang > 0.0) {
        const double k0 = th[0] / ang, k1 = th[1] / ang, k2 = th[2] / ang;
        const double s = sin(ang), cc = 1.0 - cos(ang);
        Rm[0] = 1.0 - cc * (k1 * k1 + k2 * k2);
        Rm[1] = -s * k2 + cc * k0 * k1;
        Rm[2] = s * k1 + cc * k0 * k2;
        Rm[3] = s * k2 + cc * k0 * k1;
        Rm[4] = 1.0 - cc * (k0 * k0 + k2 * k2);
        Rm[5] = -s * k0 + cc * k1 * k2;
        Rm[6] = -s * k1 + cc * k0 * k2;
        Rm[7] = s * k0 + cc * k1 * k2;
        Rm[8] = 1.0 - cc * (k0 * k0 + k1 * k1);
    }
    const double c[3] = {bpos[3 * (size_t)b], bpos[3 * (size_t)b + 1], bpos[3 * (size_t)b + 2]};
    const double nc[3] = {c[0] + dR[0], c[1] + dR[1], c[2] + dR[2]};
    for (int k = start[b] + lane; k < start[b + 1]; k += 32) {
        const int i = members[k];
        const double r[3] = {mimg(pos[3 * (size_t)i] - c[0], a.L[0]), mimg(pos[3 * (size_t)i + 1] - c[1], a.L[1]),
                             mimg(pos[3 * (size_t)i + 2] - c[2], a.L[2])};
        for (int d = 0; d < 3; ++d) {
            const double rr = Rm[3 * d] * r[0] + Rm[3 * d + 1] * r[1] + Rm[3 * d + 2] * r[2];
            pos[3 * (size_t)i + d] = wrapc(nc[d] + rr, a.L[d]);
        }
    }
    __syncwarp();
    if (lane == 0) {
        for (int d = 0; d < 3; ++d) bpos[3 * (size_t)b + d] = wrapc(nc[d], a.L[d]);
        if (moves) {
            moves[2 * (size_t)b] = sqrt(dR[0] * dR[0] + dR[1] * dR[1] + dR[2] * dR[2]);
            moves[2 * (size_t)b + 1] = ang;
        }
    }
}

}  // namespace

int body_force_torque(cr_handle *h, const double *pos, const double *bpos, const double *force, double *bf,
                      double *bt) {
    if (h->B == 0) return CR_OK;
    body_force_torque_kernel<<<blocks_for((long)h->B * 32, 256), 256, 0, h->stream>>>(
        h->B, h->d_body_start, h->d_body_members, pos, bpos, force, h->L[0], h->L[1], h->L[2], bf, bt);
    CR_LAUNCH(h, "body_force_torque_kernel");
    return CR_OK;
}

int brownian_step(cr_handle *h, const cr_brownian_params *bp, long long step, const double *radius,
                  const double *force, double *pos, double *bpos) {
    if (h->B == 0) return CR_OK;
    if (!h->d_bf) {
        CR_TRY(dalloc(h, &h->d_bf, 3 * (size_t)h->B));
        CR_TRY(dalloc(h, &h->d_bt, 3 * (size_t)h->B));
        CR_TRY(dalloc(h, &h->d_moves, 2 * (size_t)h->B));
    }
    CR_TRY(body_force_torque(h, pos, bpos, force, h->d_bf, h->d_bt));
    if (bp->repulsion > 0.0) {
        repulsion_kernel<<<blocks_for(h->B, 256), 256, 0, h->stream>>>(h->B, bpos, radius, bp->repulsion,
                                                                       bp->contact_gap, h->L[0], h->L[1], h->L[2],
                                                                       h->d_bf);
        CR_LAUNCH(h, "repulsion_kernel");
    }
    StepArgs a;
    a.dt = bp->dt;
    a.kT = bp->kT;
    a.eta = bp->viscosity;
    a.seed = bp->seed;
    a.step = step;
    for (int d = 0; d < 3; ++d) a.L[d] = h->L[d];
    brownian_kernel<<<blocks_for((long)h->B * 32, 256), 256, 0, h->stream>>>(
        h->B, a, h->d_body_start, h->d_body_members, h->d_rigid, radius, h->d_bf, h->d_bt, pos, bpos, h->d_moves);
    CR_LAUNCH(h, "brownian_kernel");
    return CR_OK;
}

}  // namespace cr
