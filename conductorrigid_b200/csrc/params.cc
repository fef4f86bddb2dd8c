// params.cc -- host-side parameter derivation and real-space tables.
//
// Restates ConductorRigid::SetParams (ConductorRigid.cc:116-379) and the kernel
// constants of PotentialChargeMultiply (ConductorRigid.cu:912-917) in FP64.  The
// reference computes these once on the host and casts them to float; here they stay
// double and each precision path casts on upload.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/conductor_rigid.h"

namespace {
const double kPi = 3.14159265358979323846;

// Sorted 5-smooth integers (2^a 3^b 5^c) in [8, 4096] (ConductorRigid.cc:129-155).
const std::vector<int> &smooth_sizes() {
    static const std::vector<int> sizes = [] {
        std::vector<int> m;
        for (long p2 = 1; p2 <= 4096; p2 *= 2)
            for (long p3 = p2; p3 <= 4096; p3 *= 3)
                for (long p5 = p3; p5 <= 4096; p5 *= 5)
                    if (p5 >= 8) m.push_back((int)p5);
        std::sort(m.begin(), m.end());
        return m;
    }();
    return sizes;
}
}  // namespace

extern "C" int cr_derive_params(const cr_params *p, const double L[3], cr_derived *out) {
    if (!p || !L || !out) return CR_BAD_PARAM;
    if (!(p->xi > 0) || !(p->errortol > 0) || !(p->errortol < 1)) return CR_BAD_PARAM;
    for (int d = 0; d < 3; ++d)
        if (!(L[d] > 0) || p->grid[d] < 0) return CR_BAD_PARAM;
    if (p->support < 0 || p->rcut < 0) return CR_BAD_PARAM;
    cr_derived r{};
    const double root = std::sqrt(-std::log(p->errortol));
    r.rcut = p->rcut > 0 ? p->rcut : root / p->xi;                  // cc:123
    r.kcut = 2.0 * p->xi * root;                                    // cc:124
    for (int d = 0; d < 3; ++d) {
        if (p->grid[d] > 0) {
            r.grid[d] = p->grid[d];
            continue;
        }
        int n = (int)std::ceil(1.0 + L[d] * r.kcut / kPi);          // cc:125-127
        for (int m : smooth_sizes())                                 // cc:161-178
            if (n <= m) { n = m; break; }
        r.grid[d] = n;
    }
    for (int d = 0; d < 3; ++d)
        if (r.grid[d] > 4096) return CR_GRID_TOO_LARGE;             // cc:181-189
    for (int d = 0; d < 3; ++d) r.h[d] = L[d] / r.grid[d];          // cc:200
    r.support_unclamped = p->support > 0 ? p->support
                                         : (int)std::ceil(-2.0 * std::log(p->errortol) / kPi);  // cc:201
    for (int d = 0; d < 3; ++d)
        r.eta[d] = r.support_unclamped * r.h[d] * r.h[d] * p->xi * p->xi / kPi;                 // cc:202
    r.support = std::min(r.support_unclamped, std::min(r.grid[0], std::min(r.grid[1], r.grid[2])));  // cc:205-207
    r.dr = 0.001;                                                    // cc:278
    r.n_table = (int)(r.rcut / r.dr - 1);                            // cc:279
    const double xi2 = p->xi * p->xi;
    r.xiterm = 2.0 * xi2;                                            // cu:915
    r.prefac = r.xiterm * p->xi / kPi * std::sqrt(2.0 / (kPi * r.eta[0] * r.eta[1] * r.eta[2]));  // cu:916
    r.quadW = r.h[0] * r.h[1] * r.h[2];                              // cu:913
    r.selfcoeff = (1.0 - std::exp(-4.0 * xi2)) / (8.0 * kPi * std::sqrt(kPi) * p->xi) +
                  std::erfc(2.0 * p->xi) / (4.0 * kPi);              // cu:917
    // The real-space sum takes one (minimum) image per pair (ConductorRigid.cu:536),
    // which is only the whole sum when rc <= L/2; HOOMD's neighbour list refuses
    // such boxes as well.
    for (int d = 0; d < 3; ++d)
        if (r.rcut > 0.5 * L[d]) return CR_BAD_PARAM;
    if (r.n_table < 1) return CR_BAD_PARAM;
    *out = r;
    return CR_OK;
}

// ConductorRigid.cc:292-354: values at dist = (i+1) dr for i = 0..n_table, each
// entry's .y holding the next entry's .x for the linear interpolation.
extern "C" int cr_build_tables(const cr_derived *d, double xi, double *phiq, double *gradphiq) {
    if (!d || !phiq || !gradphiq || !(xi > 0) || d->n_table < 1) return CR_BAD_PARAM;
    const double xi2 = xi * xi;
    const double pi15 = std::pow(kPi, 1.5);
    const int nt = d->n_table;
    for (int i = 0; i <= nt; ++i) {
        const double r = (i + 1) * d->dr;
        const double r2 = r * r;
        const double ep = std::exp(-(r + 2) * (r + 2) * xi2);
        const double em = std::exp(-(r - 2) * (r - 2) * xi2);
        const double e0 = std::exp(-r2 * xi2);
        const double cp = std::erfc((r + 2) * xi);
        const double cm = std::erfc((r - 2) * xi);
        const double c0 = std::erfc(r * xi);
        // potential / charge (cc:311-327)
        double pe_p = -(r + 2.) / (32. * pi15 * xi * r);
        double pe_m = -(r - 2.) / (32. * pi15 * xi * r);
        double pe_0 = 1. / (16. * pi15 * xi);
        double pc_p = 1. / (64. * kPi * xi2 * r) * (2. * xi2 * (r + 2.) * (r + 2.) + 1.);
        double pc_m = 1. / (64. * kPi * xi2 * r) * (2. * xi2 * (r - 2.) * (r - 2.) + 1.);
        double pc_0 = -(2. * xi2 * r2 + 1.) / (32. * kPi * xi2 * r);
        double reg = r < 2 ? -1. / (4. * kPi * r) + (4. - r) / (16. * kPi) : 0.;
        phiq[2 * i] = pe_p * ep + pe_m * em + pe_0 * e0 + pc_p * cp + pc_m * cm + pc_0 * c0 + reg;
        // its radial derivative (cc:330-345)
        pe_p = -(r - 2.) / (32. * pi15 * xi * r2);
        pe_m = -(r + 2.) / (32. * pi15 * xi * r2);
        pe_0 = 1. / (16. * pi15 * xi * r);
        pc_p = (2. * xi2 * r2 - 8. * xi2 - 1.) / (64. * kPi * xi2 * r2);
        pc_m = (2. * xi2 * r2 - 8. * xi2 - 1.) / (64. * kPi * xi2 * r2);
        pc_0 = -(2. * xi2 * r2 - 1.) / (32. * kPi * xi2 * r2);
        reg = r < 2 ? 1. / (4. * kPi * r2) - 1. / (16. * kPi) : 0.;
        gradphiq[2 * i] = pe_p * ep + pe_m * em + pe_0 * e0 + pc_p * cp + pc_m * cm + pc_0 * c0 + reg;
    }
    for (int i = 0; i < nt; ++i) {                                   // cc:350-354
        phiq[2 * i + 1] = phiq[2 * (i + 1)];
        gradphiq[2 * i + 1] = gradphiq[2 * (i + 1)];
    }
    phiq[2 * nt + 1] = 0.0;  // never read: the index stays below n_table
    gradphiq[2 * nt + 1] = 0.0;
    return CR_OK;
}
