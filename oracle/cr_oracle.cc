// cr_oracle.cc -- FP64 CPU restatement of ConductorRigid's induced-charge solve.
//
// TEST INFRASTRUCTURE ONLY (see cr_oracle.h): the checker for the CUDA product and
// the timed CPU baseline.  Parity unpinned against reference outputs (the reference
// cannot be built or run here); pinned by the known-answer tests in tests/.
//
// Compiled with -ffp-contract=off so that the neighbour-list distances match the
// product's GPU builder bit for bit.
#include "cr_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double PI = 3.14159265358979323846;
typedef std::complex<double> cplx;

// ---------------------------------------------------------------------------
// Mixed-radix FFT (own implementation; the reference uses cuFFT C2C,
// ConductorRigid.cc:228, ConductorRigid.cu:927,933).  Recursive decimation in
// time over the prime factors of n; unnormalised; sign -1 forward.
// ---------------------------------------------------------------------------
struct Fft1d {
    int n = 0;
    std::vector<int> factors;
    std::vector<cplx> tw;
    Fft1d(int n_, int sign) : n(n_) {
        int m = n;
        for (int f : {4, 2, 3, 5}) {
            while (m % f == 0) { factors.push_back(f); m /= f; }
        }
        for (int f = 7; m > 1; f += 2) {
            while (m % f == 0) { factors.push_back(f); m /= f; }
        }
        tw.resize(n);
        for (int e = 0; e < n; ++e) {
            double a = 2.0 * PI * (double)e / (double)n;
            tw[e] = cplx(std::cos(a), sign * std::sin(a));
        }
    }
    void rec(const cplx *in, cplx *out, int len, int stride, size_t fi, cplx *tmp) const {
        if (len == 1) { out[0] = in[0]; return; }
        int p = factors[fi];
        int m = len / p;
        for (int q = 0; q < p; ++q) rec(in + (size_t)q * stride, out + (size_t)q * m, m, stride * p, fi + 1, tmp);
        size_t step = (size_t)(n / len);     // w_len = w_n^{step}
        size_t pstep = (size_t)(n / p);      // w_p = w_n^{pstep}
        for (int k = 0; k < m; ++k) {
            for (int q = 0; q < p; ++q) tmp[q] = out[(size_t)q * m + k] * tw[((size_t)q * k * step) % n];
            for (int s = 0; s < p; ++s) {
                cplx acc = 0;
                for (int q = 0; q < p; ++q) acc += tmp[q] * tw[((size_t)q * s * pstep) % n];
                out[k + (size_t)m * s] = acc;
            }
        }
    }
    void run(cplx *data, cplx *work, cplx *tmp) const {
        rec(data, work, n, 1, 0, tmp);
        std::copy(work, work + n, data);
    }
};

void fft_axis(int n0, int n1, int n2, cplx *a, int axis, int sign) {
    int n = axis == 0 ? n0 : (axis == 1 ? n1 : n2);
    Fft1d f(n, sign);
    long lines = (long)n0 * n1 * n2 / n;
#pragma omp parallel
    {
        std::vector<cplx> buf(n), work(n), tmp(64 > n ? 64 : n);
#pragma omp for schedule(static)
        for (long l = 0; l < lines; ++l) {
            size_t base, stride;
            if (axis == 2) { base = (size_t)l * n2; stride = 1; }
            else if (axis == 1) { size_t i = l / n2, k = l % n2; base = i * (size_t)n1 * n2 + k; stride = n2; }
            else { base = (size_t)l; stride = (size_t)n1 * n2; }
            for (int t = 0; t < n; ++t) buf[t] = a[base + t * stride];
            f.run(buf.data(), work.data(), tmp.data());
            for (int t = 0; t < n; ++t) a[base + t * stride] = buf[t];
        }
    }
}

inline double wrapd(double x, double L) { return x - L * std::rint(x * (1.0 / L)); }

// Spreading window of one bead along one dimension (ConductorRigid.cu:193-216):
// fractional position (pos - lo)/L with lo = -L/2, scaled to grid units, the node
// immediately preceding it, and the first window node per the parity rule.
inline int window_start(double pos, double L, int N, int P, double *u_out) {
    double frac = (pos + 0.5 * L) / L;   // BoxDim::makeFraction for an orthorhombic box
    double u = frac * (double)N;
    int x = (int)u;                      // int() truncation (cu:202)
    int halfP = P / 2;
    int start = x - halfP + 1 - (P % 2) * ((u - (double)x) < 0.5 ? 1 : 0);  // cu:207-210
    if (u_out) *u_out = u;
    return start;
}
inline int wrap_index(int i, int N) { return i < 0 ? i + N : (i > N - 1 ? i - N : i); }  // cu:226-228

// Per-dimension window weights exp(-xiterm r_d^2 / eta_d) for t = 0..P-1, and
// r_d = node - pos.  The reference evaluates exp of the sum over dimensions
// (cu:219-223); the product of the per-dimension factors is the same number.
void window_1d(const orc_params *p, int d, double pos, int *idx, double *w, double *r) {
    int start = window_start(pos, p->L[d], p->N[d], p->P, nullptr);
    for (int t = 0; t < p->P; ++t) {
        int node = start + t;
        double rg = p->h[d] * node - 0.5 * p->L[d] - pos;  // cu:214-219
        idx[t] = wrap_index(node, p->N[d]);
        w[t] = std::exp(-p->xiterm * rg * rg / p->eta[d]);
        if (r) r[t] = rg;
    }
}

}  // namespace

extern "C" {

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ConductorRigid.cc:116-207 and cu:912-917.
int orc_derive(orc_params *p) {
    if (!(p->xi > 0) || !(p->errortol > 0) || !(p->errortol < 1)) return ORC_BAD_INPUT;
    for (int d = 0; d < 3; ++d) if (!(p->L[d] > 0)) return ORC_BAD_INPUT;
    double lt = std::sqrt(-std::log(p->errortol));
    p->rc = p->rc_override > 0 ? p->rc_override : lt / p->xi;     // cc:123
    p->kcut = 2.0 * p->xi * lt;                                     // cc:124
    // 5-smooth sizes in [8, 4096] (cc:129-155)
    std::vector<int> M;
    for (int a = 0; a < 13; ++a) for (int b = 0; b < 8; ++b) for (int c = 0; c < 6; ++c) {
        long m = 1;
        for (int i = 0; i < a; ++i) m *= 2;
        for (int i = 0; i < b; ++i) m *= 3;
        for (int i = 0; i < c; ++i) m *= 5;
        if (m >= 8 && m <= 4096) M.push_back((int)m);
    }
    std::sort(M.begin(), M.end());
    for (int d = 0; d < 3; ++d) {
        if (p->grid_override[d] > 0) { p->N[d] = p->grid_override[d]; continue; }
        int n = (int)std::ceil(1.0 + p->L[d] * p->kcut / PI);       // cc:125-127
        for (int m : M) if (n <= m) { n = m; break; }                // cc:161-178
        p->N[d] = n;
    }
    for (int d = 0; d < 3; ++d) if (p->N[d] > 4096) return ORC_GRID_TOO_LARGE;  // cc:181-189
    for (int d = 0; d < 3; ++d) p->h[d] = p->L[d] / p->N[d];                    // cc:200
    p->P_unclamped = p->support_override > 0 ? p->support_override
                                             : (int)std::ceil(-2.0 * std::log(p->errortol) / PI);  // cc:201
    for (int d = 0; d < 3; ++d) p->eta[d] = p->P_unclamped * p->h[d] * p->h[d] * p->xi * p->xi / PI;  // cc:202
    p->P = p->P_unclamped;
    for (int d = 0; d < 3; ++d) if (p->P > p->N[d]) p->P = p->N[d];             // cc:205-207
    p->dr = 0.001;                                                             // cc:278
    p->N_table = (int)(p->rc / p->dr - 1);                                     // cc:279
    double xi2 = p->xi * p->xi;
    p->xiterm = 2.0 * xi2;                                                     // cu:915
    p->prefac = p->xiterm * p->xi / PI * std::sqrt(2.0 / (PI * p->eta[0] * p->eta[1] * p->eta[2]));  // cu:916
    p->quadW = p->h[0] * p->h[1] * p->h[2];                                    // cu:913
    p->selfcoeff = (1.0 - std::exp(-4.0 * xi2)) / (8.0 * PI * std::sqrt(PI) * p->xi) +
                   std::erfc(2.0 * p->xi) / (4.0 * PI);                        // cu:917
    for (int d = 0; d < 3; ++d) if (p->rc > 0.5 * p->L[d]) return ORC_RC_TOO_LARGE;
    return ORC_OK;
}

// ConductorRigid.cc:292-354.
void orc_tables(const orc_params *p, double *phiq, double *gradphiq) {
    const double xi = p->xi, xi2 = xi * xi;
    const int NT = p->N_table;
    for (int i = 0; i <= NT; ++i) {
        double dist = (i + 1) * p->dr;
        double dist2 = dist * dist;
        double expp = std::exp(-(dist + 2) * (dist + 2) * xi2);
        double expm = std::exp(-(dist - 2) * (dist - 2) * xi2);
        double exp0 = std::exp(-dist2 * xi2);
        double erfp = std::erfc((dist + 2) * xi);
        double erfm = std::erfc((dist - 2) * xi);
        double erf0 = std::erfc(dist * xi);
        double pi15 = std::pow(PI, 1.5);
        double exppolyp = -(dist + 2.) / (32. * pi15 * xi * dist);
        double exppolym = -(dist - 2.) / (32. * pi15 * xi * dist);
        double exppoly0 = 1. / (16. * pi15 * xi);
        double erfpolyp = 1. / (64. * PI * xi2 * dist) * (2. * xi2 * (dist + 2.) * (dist + 2.) + 1.);
        double erfpolym = 1. / (64. * PI * xi2 * dist) * (2. * xi2 * (dist - 2.) * (dist - 2.) + 1.);
        double erfpoly0 = -(2. * xi2 * dist2 + 1.) / (32. * PI * xi2 * dist);
        double regpoly = dist < 2 ? -1. / (4. * PI * dist) + (4. - dist) / (16. * PI) : 0.;
        phiq[2 * i] = exppolyp * expp + exppolym * expm + exppoly0 * exp0 + erfpolyp * erfp +
                      erfpolym * erfm + erfpoly0 * erf0 + regpoly;
        exppolyp = -(dist - 2.) / (32. * pi15 * xi * dist2);
        exppolym = -(dist + 2.) / (32. * pi15 * xi * dist2);
        exppoly0 = 1. / (16. * pi15 * xi * dist);
        erfpolyp = (2. * xi2 * dist2 - 8. * xi2 - 1.) / (64. * PI * xi2 * dist2);
        erfpolym = (2. * xi2 * dist2 - 8. * xi2 - 1.) / (64. * PI * xi2 * dist2);
        erfpoly0 = -(2. * xi2 * dist2 - 1.) / (32. * PI * xi2 * dist2);
        regpoly = dist < 2 ? 1. / (4. * PI * dist2) - 1. / (16. * PI) : 0.;
        gradphiq[2 * i] = exppolyp * expp + exppolym * expm + exppoly0 * exp0 + erfpolyp * erfp +
                          erfpolym * erfm + erfpoly0 * erf0 + regpoly;
    }
    for (int i = 0; i < NT; ++i) {            // cc:350-354
        phiq[2 * i + 1] = phiq[2 * (i + 1)];
        gradphiq[2 * i + 1] = gradphiq[2 * (i + 1)];
    }
    phiq[2 * NT + 1] = 0.0;                   // never read (the index stays below N_table)
    gradphiq[2 * NT + 1] = 0.0;
}

// ConductorRigid.cc:245-274.
void orc_scale(const orc_params *p, double *scale) {
    const int Nx = p->N[0], Ny = p->N[1], Nz = p->N[2];
    const double Ng = (double)Nx * Ny * Nz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < Nz; ++k) {
                size_t idx = ((size_t)i * Ny + j) * Nz + k;
                double kx = ((i < (Nx + 1) / 2) ? i : i - Nx) * 2.0 * PI / p->L[0];
                double ky = ((j < (Ny + 1) / 2) ? j : j - Ny) * 2.0 * PI / p->L[1];
                double kz = ((k < (Nz + 1) / 2) ? k : k - Nz) * 2.0 * PI / p->L[2];
                double k2 = kx * kx + ky * ky + kz * kz;
                double etak2 = (1.0 - p->eta[0]) * kx * kx + (1.0 - p->eta[1]) * ky * ky +
                               (1.0 - p->eta[2]) * kz * kz;
                if (i == 0 && j == 0 && k == 0) { scale[idx] = 0.0; continue; }
                double kk = std::sqrt(k2);
                double j0 = std::sin(kk) / kk;
                scale[idx] = j0 * j0 * std::exp(-etak2 / (4.0 * p->xi * p->xi)) / k2 / Ng;
            }
}

void orc_fft3d(int n0, int n1, int n2, double *re, double *im, int sign) {
    size_t G = (size_t)n0 * n1 * n2;
    std::vector<cplx> a(G);
    for (size_t i = 0; i < G; ++i) a[i] = cplx(re[i], im[i]);
    fft_axis(n0, n1, n2, a.data(), 2, sign);
    fft_axis(n0, n1, n2, a.data(), 1, sign);
    fft_axis(n0, n1, n2, a.data(), 0, sign);
    for (size_t i = 0; i < G; ++i) { re[i] = a[i].real(); im[i] = a[i].imag(); }
}

// ConductorRigid.cu:144-234.  Race-free: each thread owns a slab of x-planes and
// adds the contributions of every bead whose window reaches into it.
void orc_spread(const orc_params *p, int N, const double *pos, const double *q, double *grid) {
    const int Nx = p->N[0], Ny = p->N[1], Nz = p->N[2], P = p->P;
    size_t G = (size_t)Nx * Ny * Nz;
    std::fill(grid, grid + G, 0.0);
#pragma omp parallel
    {
        int nt = 1, tid = 0;
#ifdef _OPENMP
        nt = omp_get_num_threads();
        tid = omp_get_thread_num();
#endif
        int x0 = (int)((long)Nx * tid / nt), x1 = (int)((long)Nx * (tid + 1) / nt);
        std::vector<int> ix(P), iy(P), iz(P);
        std::vector<double> wx(P), wy(P), wz(P);
        for (int n = 0; n < N; ++n) {
            window_1d(p, 0, pos[3 * n + 0], ix.data(), wx.data(), nullptr);
            bool hit = false;
            for (int t = 0; t < P; ++t) hit |= (ix[t] >= x0 && ix[t] < x1);
            if (!hit) continue;
            window_1d(p, 1, pos[3 * n + 1], iy.data(), wy.data(), nullptr);
            window_1d(p, 2, pos[3 * n + 2], iz.data(), wz.data(), nullptr);
            double c = p->prefac * q[n];
            for (int a = 0; a < P; ++a) {
                if (ix[a] < x0 || ix[a] >= x1) continue;
                for (int b = 0; b < P; ++b) {
                    double cab = c * wx[a] * wy[b];
                    double *row = grid + ((size_t)ix[a] * Ny + iy[b]) * Nz;
                    for (int t = 0; t < P; ++t) row[iz[t]] += cab * wz[t];
                }
            }
        }
    }
}

// ConductorRigid.cu:260-360 (prefactor quadW*prefac, cu:936-937).
void orc_contract(const orc_params *p, int N, const double *pos, const double *grid, double *phi) {
    const int Ny = p->N[1], Nz = p->N[2], P = p->P;
    const double c = p->quadW * p->prefac;
#pragma omp parallel
    {
        std::vector<int> ix(P), iy(P), iz(P);
        std::vector<double> wx(P), wy(P), wz(P);
#pragma omp for schedule(static)
        for (int n = 0; n < N; ++n) {
            window_1d(p, 0, pos[3 * n + 0], ix.data(), wx.data(), nullptr);
            window_1d(p, 1, pos[3 * n + 1], iy.data(), wy.data(), nullptr);
            window_1d(p, 2, pos[3 * n + 2], iz.data(), wz.data(), nullptr);
            double acc = 0.0;
            for (int a = 0; a < P; ++a)
                for (int b = 0; b < P; ++b) {
                    const double *row = grid + ((size_t)ix[a] * Ny + iy[b]) * Nz;
                    double s = 0.0;
                    for (int t = 0; t < P; ++t) s += wz[t] * row[iz[t]];
                    acc += wx[a] * wy[b] * s;
                }
            phi[n] = c * acc;
        }
    }
}

// ConductorRigid.cu:363-466 (prefactor quadW*prefac, cu:1273-1274); r = pos - node.
void orc_contract_force(const orc_params *p, int N, const double *pos, const double *q,
                        const double *grid, double *force) {
    const int Ny = p->N[1], Nz = p->N[2], P = p->P;
    const double c = 2.0 * p->quadW * p->prefac * p->xiterm;
#pragma omp parallel
    {
        std::vector<int> ix(P), iy(P), iz(P);
        std::vector<double> wx(P), wy(P), wz(P), rx(P), ry(P), rz(P);
#pragma omp for schedule(static)
        for (int n = 0; n < N; ++n) {
            window_1d(p, 0, pos[3 * n + 0], ix.data(), wx.data(), rx.data());
            window_1d(p, 1, pos[3 * n + 1], iy.data(), wy.data(), ry.data());
            window_1d(p, 2, pos[3 * n + 2], iz.data(), wz.data(), rz.data());
            double fx = 0, fy = 0, fz = 0;
            for (int a = 0; a < P; ++a)
                for (int b = 0; b < P; ++b) {
                    const double *row = grid + ((size_t)ix[a] * Ny + iy[b]) * Nz;
                    double s0 = 0.0, s1 = 0.0;
                    for (int t = 0; t < P; ++t) {
                        double g = wz[t] * row[iz[t]];
                        s0 += g;
                        s1 += g * (-rz[t]) / p->eta[2];  // r = pos - node = -(node - pos)
                    }
                    double wab = wx[a] * wy[b];
                    fx += wab * s0 * (-rx[a]) / p->eta[0];
                    fy += wab * s0 * (-ry[b]) / p->eta[1];
                    fz += wab * s1;
                }
            force[3 * n + 0] = c * q[n] * fx;
            force[3 * n + 1] = c * q[n] * fy;
            force[3 * n + 2] = c * q[n] * fz;
        }
    }
}

static void wave_grid(const orc_params *p, int N, const double *pos, const double *q,
                      std::vector<double> &grid) {
    const int Nx = p->N[0], Ny = p->N[1], Nz = p->N[2];
    size_t G = (size_t)Nx * Ny * Nz;
    grid.assign(G, 0.0);
    orc_spread(p, N, pos, q, grid.data());          // cu:923
    std::vector<double> im(G, 0.0), sc(G);
    orc_fft3d(Nx, Ny, Nz, grid.data(), im.data(), -1);   // cu:927
    orc_scale(p, sc.data());
    for (size_t i = 0; i < G; ++i) { grid[i] *= sc[i]; im[i] *= sc[i]; }  // cu:930
    orc_fft3d(Nx, Ny, Nz, grid.data(), im.data(), +1);   // cu:933 (real part used)
}

void orc_wave_potential(const orc_params *p, int N, const double *pos, const double *q, double *phi) {
    std::vector<double> grid;
    wave_grid(p, N, pos, q, grid);
    orc_contract(p, N, pos, grid.data(), phi);      // cu:936
}

void orc_wave_force(const orc_params *p, int N, const double *pos, const double *q, double *force) {
    std::vector<double> grid;
    wave_grid(p, N, pos, q, grid);
    orc_contract_force(p, N, pos, q, grid.data(), force);  // cu:1273
}

// Cell-list neighbour search (the reference takes HOOMD's NeighborListGPUBinned,
// compute.py:38-44, with no exclusions).  Same pair set: every j != i whose
// minimum-image distance is below r_list.
int64_t orc_neighbor_list(int N, const double *pos, const double L[3], double r_list,
                          int *count, int64_t *head, int *list) {
    int nc[3];
    for (int d = 0; d < 3; ++d) nc[d] = std::max(1, (int)std::floor(L[d] / r_list));
    bool brute = nc[0] < 3 || nc[1] < 3 || nc[2] < 3;
    const double rl2 = r_list * r_list;
    auto cell_of = [&](int i, int d) {
        double f = (pos[3 * i + d] + 0.5 * L[d]) / L[d];
        int c = (int)std::floor(f * nc[d]);
        return ((c % nc[d]) + nc[d]) % nc[d];
    };
    std::vector<int> cstart, cbeads;
    if (!brute) {
        size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
        std::vector<int> cnt(ncell + 1, 0), cid(N);
        for (int i = 0; i < N; ++i) {
            cid[i] = (cell_of(i, 0) * nc[1] + cell_of(i, 1)) * nc[2] + cell_of(i, 2);
            cnt[cid[i] + 1]++;
        }
        for (size_t c = 0; c < ncell; ++c) cnt[c + 1] += cnt[c];
        cstart = cnt;
        cbeads.resize(N);
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (int i = 0; i < N; ++i) cbeads[fill[cid[i]]++] = i;
    }
    auto d2_of = [&](int i, int j) {
        double dx = wrapd(pos[3 * i + 0] - pos[3 * j + 0], L[0]);
        double dy = wrapd(pos[3 * i + 1] - pos[3 * j + 1], L[1]);
        double dz = wrapd(pos[3 * i + 2] - pos[3 * j + 2], L[2]);
        return dx * dx + dy * dy + dz * dz;
    };
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (int i = 0; i < N; ++i) {
        std::vector<int> nb;
        if (brute) {
            for (int j = 0; j < N; ++j) if (j != i && d2_of(i, j) < rl2) nb.push_back(j);
        } else {
            int ci[3] = {cell_of(i, 0), cell_of(i, 1), cell_of(i, 2)};
            for (int a = -1; a <= 1; ++a) for (int b = -1; b <= 1; ++b) for (int c = -1; c <= 1; ++c) {
                int x = (ci[0] + a + nc[0]) % nc[0], y = (ci[1] + b + nc[1]) % nc[1], z = (ci[2] + c + nc[2]) % nc[2];
                size_t cell = ((size_t)x * nc[1] + y) * nc[2] + z;
                for (int k = cstart[cell]; k < cstart[cell + 1]; ++k) {
                    int j = cbeads[k];
                    if (j != i && d2_of(i, j) < rl2) nb.push_back(j);
                }
            }
            std::sort(nb.begin(), nb.end());
        }
        count[i] = (int)nb.size();
        total += (int64_t)nb.size();
        if (list) std::copy(nb.begin(), nb.end(), list + head[i]);
    }
    if (head && !list) {
        int64_t s = 0;
        for (int i = 0; i < N; ++i) { head[i] = s; s += count[i]; }
    }
    return total;
}

// Table lookup and linear interpolation (ConductorRigid.cu:549-554).
static inline double table_lerp(const orc_params *p, const double *T, double dist) {
    int ind = (int)std::floor(p->N_table * (dist - p->dr) / (p->rc - p->dr));
    double lin = dist / p->dr - ind - 1.0;
    double x = T[2 * ind], y = T[2 * ind + 1];
    return x + (y - x) * lin;
}

// ConductorRigid.cu:469-567 (without the final Phi_b - phi, done in orc_matvec).
void orc_real_space(const orc_params *p, int N, const double *pos, const double *q,
                    const double *phiq_table, const int64_t *head, const int *count,
                    const int *list, double *phi_io) {
    const double rc2 = p->rc * p->rc, rmin2 = p->dr * p->dr;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < N; ++i) {
        double phi = phi_io[i] + p->selfcoeff * q[i];   // cu:506
        for (int k = 0; k < count[i]; ++k) {
            int j = list[head[i] + k];
            double dx = wrapd(pos[3 * i + 0] - pos[3 * j + 0], p->L[0]);
            double dy = wrapd(pos[3 * i + 1] - pos[3 * j + 1], p->L[1]);
            double dz = wrapd(pos[3 * i + 2] - pos[3 * j + 2], p->L[2]);
            double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 < rc2 && d2 >= rmin2) phi += table_lerp(p, phiq_table, std::sqrt(d2)) * q[j];  // cu:540-557
        }
        phi_io[i] = phi;
    }
}

// ConductorRigid.cu:570-664.
void orc_real_space_force(const orc_params *p, int N, const double *pos, const double *q,
                          const double E0[3], const double *gradphiq_table,
                          const int64_t *head, const int *count, const int *list,
                          double *force_io) {
    const double rc2 = p->rc * p->rc, rmin2 = p->dr * p->dr;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < N; ++i) {
        double qi = q[i];
        double F[3] = {force_io[3 * i] + qi * E0[0], force_io[3 * i + 1] + qi * E0[1],
                       force_io[3 * i + 2] + qi * E0[2]};          // cu:603
        for (int k = 0; k < count[i]; ++k) {
            int j = list[head[i] + k];
            double r[3];
            for (int d = 0; d < 3; ++d) r[d] = wrapd(pos[3 * i + d] - pos[3 * j + d], p->L[d]);
            double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            if (d2 < rc2 && d2 >= rmin2) {
                double dist = std::sqrt(d2);
                double A = table_lerp(p, gradphiq_table, dist);
                for (int d = 0; d < 3; ++d) F[d] += -A * qi * q[j] * (r[d] / dist);  // cu:654
            }
        }
        for (int d = 0; d < 3; ++d) force_io[3 * i + d] = F[d];
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Solver context.
// ---------------------------------------------------------------------------
struct orc_ctx {
    orc_params p;
    int N, B;
    std::vector<uint32_t> body;
    std::vector<uint8_t> rigid;
    std::vector<double> Q;
    std::vector<int> bsize;
    std::vector<double> phiq, gradphiq;
    std::vector<double> pos, bpos;
    std::vector<int> count, list;
    std::vector<int64_t> head;
};

extern "C" {

orc_ctx *orc_create(const orc_params *p, int N, int B, const uint32_t *body, const uint8_t *rigid,
                    const double *body_charge) {
    orc_ctx *c = new orc_ctx();
    c->p = *p;
    c->N = N;
    c->B = B;
    c->body.assign(body, body + N);
    c->rigid.assign(rigid, rigid + B);
    c->Q.assign(body_charge, body_charge + B);
    c->bsize.assign(B, 0);
    for (int i = 0; i < N; ++i) c->bsize[body[i]]++;
    c->phiq.resize(2 * (size_t)(p->N_table + 1));
    c->gradphiq.resize(2 * (size_t)(p->N_table + 1));
    orc_tables(p, c->phiq.data(), c->gradphiq.data());
    return c;
}

void orc_destroy(orc_ctx *c) { delete c; }

int orc_set_positions(orc_ctx *c, const double *pos, const double *body_pos) {
    c->pos.assign(pos, pos + 3 * (size_t)c->N);
    c->bpos.assign(body_pos, body_pos + 3 * (size_t)c->B);
    c->count.assign(c->N, 0);
    c->head.assign(c->N, 0);
    int64_t tot = orc_neighbor_list(c->N, pos, c->p.L, c->p.rc, c->count.data(), c->head.data(), nullptr);
    c->list.assign((size_t)tot, 0);
    orc_neighbor_list(c->N, pos, c->p.L, c->p.rc, c->count.data(), c->head.data(), c->list.data());
    return ORC_OK;
}

void orc_apply_M(orc_ctx *c, const double *q, double *Mq) {
    orc_wave_potential(&c->p, c->N, c->pos.data(), q, Mq);
    orc_real_space(&c->p, c->N, c->pos.data(), q, c->phiq.data(), c->head.data(), c->count.data(),
                   c->list.data(), Mq);
}

// ConductorRigid.cu:953-1020: top rows Phi_b - M q (cu:564), bottom rows the body
// charge sums (sum_charges cu:667-730 for rigid bodies, set_charge cu:733-761 for
// free beads; both are the sum over the body's members).
void orc_matvec(orc_ctx *c, const double *x, double *y) {
    const int N = c->N, B = c->B;
    std::vector<double> Mq(N);
    orc_apply_M(c, x, Mq.data());
    for (int i = 0; i < N; ++i) y[i] = x[N + c->body[i]] - Mq[i];
    for (int b = 0; b < B; ++b) y[N + b] = 0.0;
    for (int i = 0; i < N; ++i) y[N + c->body[i]] += x[i];
}

// ConductorRigid.cu:816-859.  The reference writes the rigid-body rows twice
// (1/(4 pi) by the row's own thread, 1/size by the rigid body's thread, cu:837,855);
// the intended and (for rigid index == body tag) actual result is 1/size.
void orc_precondition(orc_ctx *c, const double *x, double *y) {
    const int N = c->N, B = c->B;
    for (int i = 0; i < N; ++i) y[i] = -4.0 * PI * x[i];
    for (int b = 0; b < B; ++b) y[N + b] = c->rigid[b] ? x[N + b] / c->bsize[b] : x[N + b] / (4.0 * PI);
}

// ConductorRigid.cu:764-813 (free beads keep the zero from zero_array, cu:1102).
void orc_objective(orc_ctx *c, const double E0[3], double *rhs) {
    const int N = c->N, B = c->B;
    for (int i = 0; i < N; ++i) {
        uint32_t b = c->body[i];
        if (!c->rigid[b]) { rhs[i] = 0.0; continue; }
        double r[3];
        for (int d = 0; d < 3; ++d) r[d] = wrapd(c->pos[3 * i + d] - c->bpos[3 * b + d], c->p.L[d]);
        rhs[i] = -(r[0] * E0[0] + r[1] * E0[1] + r[2] * E0[2]);
    }
    for (int b = 0; b < B; ++b) rhs[N + b] = c->Q[b];
}

static double nrm2(const std::vector<double> &v) {
    double s = 0;
    for (double a : v) s += a * a;
    return std::sqrt(s);
}

// Restarted, left-preconditioned GMRES with the stopping rule of CUSP's
// default_monitor (relative tolerance times ||b||, iteration limit), as called
// at ConductorRigid.cu:1134-1136 with restart 10 and limit 100.  CUSP itself is
// not vendored; this is the textbook algorithm (Saad, "Iterative Methods for
// Sparse Linear Systems", Alg. 6.9 with Givens rotations).
int orc_gmres(orc_ctx *c, double *x, const double *b, int restart, int maxiter, double tol,
              double *resid_out, double *true_rel) {
    const int n = c->N + c->B;
    const int R = restart;
    std::vector<double> bb(b, b + n);
    const double bnorm = nrm2(bb);
    const double target = tol * bnorm;
    std::vector<std::vector<double>> V(R + 1, std::vector<double>(n));
    std::vector<double> H((size_t)(R + 1) * R), cs(R), sn(R), s(R + 1);
    std::vector<double> w(n), t(n);
    int iters = 0;
    double resid = 0;
    for (;;) {
        orc_matvec(c, x, t.data());
        for (int i = 0; i < n; ++i) t[i] = bb[i] - t[i];
        orc_precondition(c, t.data(), w.data());
        double beta = nrm2(w);
        resid = beta;
        if (beta <= target || iters >= maxiter || beta == 0.0) break;
        for (int i = 0; i < n; ++i) V[0][i] = w[i] / beta;
        std::fill(s.begin(), s.end(), 0.0);
        s[0] = beta;
        int j = 0;
        for (; j < R && iters < maxiter; ++j) {
            ++iters;
            orc_matvec(c, V[j].data(), t.data());
            orc_precondition(c, t.data(), w.data());
            for (int k = 0; k <= j; ++k) {  // modified Gram-Schmidt
                double h = 0;
                for (int i = 0; i < n; ++i) h += w[i] * V[k][i];
                H[(size_t)k * R + j] = h;
                for (int i = 0; i < n; ++i) w[i] -= h * V[k][i];
            }
            double hn = nrm2(w);
            H[(size_t)(j + 1) * R + j] = hn;
            for (int i = 0; i < n; ++i) V[j + 1][i] = hn > 0 ? w[i] / hn : 0.0;
            for (int k = 0; k < j; ++k) {
                double a = H[(size_t)k * R + j], bk = H[(size_t)(k + 1) * R + j];
                H[(size_t)k * R + j] = cs[k] * a + sn[k] * bk;
                H[(size_t)(k + 1) * R + j] = -sn[k] * a + cs[k] * bk;
            }
            double a = H[(size_t)j * R + j], bk = H[(size_t)(j + 1) * R + j];
            double den = std::sqrt(a * a + bk * bk);
            cs[j] = den > 0 ? a / den : 1.0;
            sn[j] = den > 0 ? bk / den : 0.0;
            H[(size_t)j * R + j] = den;
            H[(size_t)(j + 1) * R + j] = 0.0;
            s[j + 1] = -sn[j] * s[j];
            s[j] = cs[j] * s[j];
            resid = std::fabs(s[j + 1]);
            if (resid <= target || hn == 0.0) { ++j; break; }
        }
        // back substitution and update x += V y
        std::vector<double> y(j);
        for (int r = j - 1; r >= 0; --r) {
            double acc = s[r];
            for (int k = r + 1; k < j; ++k) acc -= H[(size_t)r * R + k] * y[k];
            y[r] = acc / H[(size_t)r * R + r];
        }
        for (int k = 0; k < j; ++k)
            for (int i = 0; i < n; ++i) x[i] += y[k] * V[k][i];
        if (resid <= target || iters >= maxiter) {
            // final preconditioned residual from x itself
            orc_matvec(c, x, t.data());
            for (int i = 0; i < n; ++i) t[i] = bb[i] - t[i];
            orc_precondition(c, t.data(), w.data());
            resid = nrm2(w);
            if (resid <= target || iters >= maxiter) break;
        }
    }
    if (resid_out) *resid_out = resid;
    if (true_rel) {
        orc_matvec(c, x, t.data());
        double r2 = 0;
        for (int i = 0; i < n; ++i) r2 += (bb[i] - t[i]) * (bb[i] - t[i]);
        *true_rel = bnorm > 0 ? std::sqrt(r2) / bnorm : std::sqrt(r2);
    }
    return iters;
}

// ConductorRigid.cu:1256-1278: wave-space force (overwrite), then q E0 plus the
// real-space gradient sum.
void orc_forces(orc_ctx *c, const double *q, const double E0[3], double *force) {
    orc_wave_force(&c->p, c->N, c->pos.data(), q, force);
    orc_real_space_force(&c->p, c->N, c->pos.data(), q, E0, c->gradphiq.data(), c->head.data(),
                         c->count.data(), c->list.data(), force);
}

// ConductorRigid.cu:1051-1151 and 1153-1286.
int orc_solve(orc_ctx *c, const double E0[3], double *q_io, double *phi_io, double *force,
              int restart, int maxiter, double tol, double *true_rel) {
    const int N = c->N, B = c->B;
    std::vector<double> rhs(N + B), x(N + B);
    orc_objective(c, E0, rhs.data());
    std::copy(q_io, q_io + N, x.begin());                 // warm start (cu:1126-1127)
    std::copy(phi_io, phi_io + B, x.begin() + N);
    double resid = 0;
    int it = orc_gmres(c, x.data(), rhs.data(), restart, maxiter, tol, &resid, true_rel);
    std::copy(x.begin(), x.begin() + N, q_io);           // cu:1139-1140
    std::copy(x.begin() + N, x.end(), phi_io);
    if (force) orc_forces(c, q_io, E0, force);
    return it;
}

}  // extern "C"
