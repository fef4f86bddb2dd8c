// systems.cc -- synthetic conductor systems (host only).
//
// Builds the inputs the benchmark workloads are defined on: icosphere surface
// beads (level 1 = 42 vertices, level 2 = 162) and random non-overlapping sphere
// centres in a periodic orthorhombic box, by random sequential addition with a
// SplitMix64 generator so that a seed fixes the system on every machine.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <utility>
#include <vector>

#include "../../include/conductor_rigid.h"

namespace {

struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace

extern "C" {

int cr_util_icosphere_count(int level) {
    if (level < 0 || level > 6) return -1;
    int n = 12;
    int e = 30, f = 20;
    for (int l = 0; l < level; ++l) {
        n += e;
        e = 2 * e + 3 * f;
        f *= 4;
    }
    return n;
}

// Unit-sphere vertices of an icosahedron subdivided `level` times (each face split
// into four at its edge midpoints, which are pushed out to the sphere).
int cr_util_icosphere(int level, double *verts) {
    int count = cr_util_icosphere_count(level);
    if (count < 0 || !verts) return CR_BAD_PARAM;
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<double> v = {-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0, 0, -1, t, 0, 1, t,
                             0, -1, -t, 0, 1, -t, t, 0, -1, t, 0, 1, -t, 0, -1, -t, 0, 1};
    std::vector<int> faces = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4,
                              11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8,
                              3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    auto normalise = [&](int i) {
        double *p = &v[3 * i];
        double r = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        p[0] /= r; p[1] /= r; p[2] /= r;
    };
    for (int i = 0; i < 12; ++i) normalise(i);
    for (int l = 0; l < level; ++l) {
        std::map<std::pair<int, int>, int> mid;
        auto midpoint = [&](int a, int b) {
            std::pair<int, int> key(std::min(a, b), std::max(a, b));
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            int idx = (int)(v.size() / 3);
            for (int d = 0; d < 3; ++d) v.push_back(0.5 * (v[3 * a + d] + v[3 * b + d]));
            normalise(idx);
            mid[key] = idx;
            return idx;
        };
        std::vector<int> nf;
        for (size_t f = 0; f < faces.size(); f += 3) {
            int a = faces[f], b = faces[f + 1], c = faces[f + 2];
            int ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            int add[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
            nf.insert(nf.end(), add, add + 12);
        }
        faces.swap(nf);
    }
    std::copy(v.begin(), v.end(), verts);
    return CR_OK;
}

// Random sequential addition of n spheres (radii[i]) with centres uniform in the
// periodic box [-L/2, L/2)^3, no two closer than the sum of their radii.  Spheres
// are inserted largest first; max_attempts bounds the total number of trials.
int cr_util_place_spheres(int n, const double *radii, const double L[3], uint64_t seed,
                          int64_t max_attempts, double *centres) {
    if (n < 0 || !radii || !L || !centres) return CR_BAD_PARAM;
    if (n == 0) return CR_OK;
    double rmax = 0;
    for (int i = 0; i < n; ++i) rmax = std::max(rmax, radii[i]);
    int nc[3];
    for (int d = 0; d < 3; ++d) nc[d] = std::max(1, (int)std::floor(L[d] / (2.0 * rmax)));
    std::vector<std::vector<int>> cells((size_t)nc[0] * nc[1] * nc[2]);
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return radii[a] > radii[b]; });
    SplitMix64 rng(seed);
    int64_t attempts = 0;
    auto cell_of = [&](const double *c, int d) {
        int k = (int)std::floor((c[d] + 0.5 * L[d]) / L[d] * nc[d]);
        return ((k % nc[d]) + nc[d]) % nc[d];
    };
    for (int oi = 0; oi < n; ++oi) {
        int i = order[oi];
        bool placed = false;
        while (!placed) {
            if (attempts++ >= max_attempts) return CR_NOT_CONVERGED;
            double c[3];
            for (int d = 0; d < 3; ++d) c[d] = (rng.uniform() - 0.5) * L[d];
            int ci[3] = {cell_of(c, 0), cell_of(c, 1), cell_of(c, 2)};
            bool ok = true;
            int span[3];
            for (int d = 0; d < 3; ++d) span[d] = nc[d] >= 3 ? 1 : 0;
            for (int a = -span[0]; a <= span[0] && ok; ++a)
                for (int b = -span[1]; b <= span[1] && ok; ++b)
                    for (int cc = -span[2]; cc <= span[2] && ok; ++cc) {
                        int x = (ci[0] + a + nc[0]) % nc[0], y = (ci[1] + b + nc[1]) % nc[1],
                            z = (ci[2] + cc + nc[2]) % nc[2];
                        for (int j : cells[((size_t)x * nc[1] + y) * nc[2] + z]) {
                            double d2 = 0;
                            for (int d = 0; d < 3; ++d) {
                                double dx = c[d] - centres[3 * j + d];
                                dx -= L[d] * std::rint(dx / L[d]);
                                d2 += dx * dx;
                            }
                            double s = radii[i] + radii[j];
                            if (d2 < s * s) { ok = false; break; }
                        }
                    }
            if (nc[0] < 3 || nc[1] < 3 || nc[2] < 3) {
                // small boxes: the cell stencil would miss or repeat images, check all
                ok = true;
                for (int oj = 0; oj < oi && ok; ++oj) {
                    int j = order[oj];
                    double d2 = 0;
                    for (int d = 0; d < 3; ++d) {
                        double dx = c[d] - centres[3 * j + d];
                        dx -= L[d] * std::rint(dx / L[d]);
                        d2 += dx * dx;
                    }
                    double s = radii[i] + radii[j];
                    if (d2 < s * s) ok = false;
                }
            }
            if (!ok) continue;
            for (int d = 0; d < 3; ++d) centres[3 * i + d] = c[d];
            cells[((size_t)ci[0] * nc[1] + ci[1]) * nc[2] + ci[2]].push_back(i);
            placed = true;
        }
    }
    return CR_OK;
}

// Uniform random doubles in [0, 1) from the same generator (used for charges,
// field directions and replica sizes so that every layer sees the same numbers).
int cr_util_uniform(uint64_t seed, int64_t n, double *out) {
    if (n < 0 || (!out && n > 0)) return CR_BAD_PARAM;
    SplitMix64 rng(seed);
    for (int64_t i = 0; i < n; ++i) out[i] = rng.uniform();
    return CR_OK;
}

}  // extern "C"
