// cr_systems.cc -- synthetic conductor systems for the oracle (TEST INFRASTRUCTURE).
//
// The oracle side builds the benchmark inputs itself, so that the CPU baseline and
// the reference-method arm run without loading the CUDA product library.  The systems
// are defined by these rules, which the product's generator follows too (a test checks
// that both give identical arrays):
//   - SplitMix64 stream (Steele, Lea, Flood 2014): state += 0x9E3779B97F4A7C15, then
//     the two xor-shift-multiply rounds; uniform doubles from the top 53 bits;
//   - icosphere: the 12 vertices (+-1, +-t, 0) cyclic with t the golden ratio,
//     normalised, 20 faces; each level splits every face into four at its edge
//     midpoints (one new vertex per edge, in order of first use), pushed to the sphere;
//   - random sequential addition: spheres in order of decreasing radius (stable),
//     trial centres (u - 1/2) L per axis, rejected when closer than the sum of radii
//     to a placed sphere (minimum image); placed spheres are binned in cells of edge
//     >= 2 r_max and only the 27 neighbouring cells are checked, or all placed spheres
//     when a box holds fewer than 3 cells along an axis.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <utility>
#include <vector>

#include "cr_oracle.h"

namespace {

uint64_t splitmix_next(uint64_t &state) {
    state += 0x9E3779B97F4A7C15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double splitmix_uniform(uint64_t &state) {
    return (double)(splitmix_next(state) >> 11) * (1.0 / 9007199254740992.0);
}

void to_unit(double *p) {
    const double r = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    p[0] /= r;
    p[1] /= r;
    p[2] /= r;
}

double min_image_dist2(const double *a, const double *b, const double L[3]) {
    double d2 = 0;
    for (int d = 0; d < 3; ++d) {
        double dx = a[d] - b[d];
        dx -= L[d] * std::rint(dx / L[d]);
        d2 += dx * dx;
    }
    return d2;
}

}  // namespace

extern "C" {

int orc_icosphere_count(int level) {
    if (level < 0 || level > 6) return -1;
    int verts = 12, edges = 30, faces = 20;
    for (int l = 0; l < level; ++l) {
        verts += edges;            // one new vertex per edge
        edges = 2 * edges + 3 * faces;
        faces *= 4;
    }
    return verts;
}

int orc_icosphere(int level, double *out) {
    const int count = orc_icosphere_count(level);
    if (count < 0 || !out) return ORC_BAD_INPUT;
    const double t = 0.5 * (1.0 + std::sqrt(5.0));
    std::vector<double> v = {-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0,
                             0, -1, t, 0, 1, t, 0, -1, -t, 0, 1, -t,
                             t, 0, -1, t, 0, 1, -t, 0, -1, -t, 0, 1};
    std::vector<int> tri = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11,
                            1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
                            3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9,
                            4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (int i = 0; i < 12; ++i) to_unit(&v[3 * i]);
    for (int l = 0; l < level; ++l) {
        std::map<std::pair<int, int>, int> edge_vertex;
        auto split = [&](int a, int b) -> int {
            const std::pair<int, int> e(std::min(a, b), std::max(a, b));
            auto found = edge_vertex.find(e);
            if (found != edge_vertex.end()) return found->second;
            const int id = (int)(v.size() / 3);
            for (int d = 0; d < 3; ++d) v.push_back(0.5 * (v[3 * a + d] + v[3 * b + d]));
            to_unit(&v[3 * id]);
            edge_vertex.emplace(e, id);
            return id;
        };
        std::vector<int> next;
        next.reserve(tri.size() * 4);
        for (size_t f = 0; f < tri.size(); f += 3) {
            const int a = tri[f], b = tri[f + 1], c = tri[f + 2];
            const int ab = split(a, b), bc = split(b, c), ca = split(c, a);
            const int four[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
            next.insert(next.end(), four, four + 12);
        }
        tri.swap(next);
    }
    std::copy(v.begin(), v.end(), out);
    return ORC_OK;
}

int orc_uniform(uint64_t seed, int64_t n, double *out) {
    if (n < 0 || (n > 0 && !out)) return ORC_BAD_INPUT;
    uint64_t state = seed;
    for (int64_t i = 0; i < n; ++i) out[i] = splitmix_uniform(state);
    return ORC_OK;
}

int orc_place_spheres(int n, const double *radii, const double L[3], uint64_t seed, int64_t max_attempts,
                      double *centres) {
    if (n < 0 || !radii || !L || !centres) return ORC_BAD_INPUT;
    if (n == 0) return ORC_OK;
    const double rmax = *std::max_element(radii, radii + n);
    int nc[3];
    for (int d = 0; d < 3; ++d) nc[d] = std::max(1, (int)std::floor(L[d] / (2.0 * rmax)));
    const bool small_box = nc[0] < 3 || nc[1] < 3 || nc[2] < 3;
    std::vector<std::vector<int>> cell((size_t)nc[0] * nc[1] * nc[2]);
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return radii[a] > radii[b]; });
    auto cell_index = [&](double x, int d) {
        const int k = (int)std::floor((x + 0.5 * L[d]) / L[d] * nc[d]);
        return ((k % nc[d]) + nc[d]) % nc[d];
    };
    uint64_t state = seed;
    int64_t tried = 0;
    for (int placed = 0; placed < n; ++placed) {
        const int i = order[placed];
        for (;;) {
            if (tried++ >= max_attempts) return ORC_BAD_INPUT;
            double c[3];
            for (int d = 0; d < 3; ++d) c[d] = (splitmix_uniform(state) - 0.5) * L[d];
            const int ci[3] = {cell_index(c[0], 0), cell_index(c[1], 1), cell_index(c[2], 2)};
            bool free_spot = true;
            if (small_box) {
                for (int k = 0; k < placed && free_spot; ++k) {
                    const int j = order[k];
                    const double s = radii[i] + radii[j];
                    if (min_image_dist2(c, centres + 3 * j, L) < s * s) free_spot = false;
                }
            } else {
                for (int a = -1; a <= 1 && free_spot; ++a)
                    for (int b = -1; b <= 1 && free_spot; ++b)
                        for (int e = -1; e <= 1 && free_spot; ++e) {
                            const int x = (ci[0] + a + nc[0]) % nc[0], y = (ci[1] + b + nc[1]) % nc[1],
                                      z = (ci[2] + e + nc[2]) % nc[2];
                            for (int j : cell[((size_t)x * nc[1] + y) * nc[2] + z]) {
                                const double s = radii[i] + radii[j];
                                if (min_image_dist2(c, centres + 3 * j, L) < s * s) {
                                    free_spot = false;
                                    break;
                                }
                            }
                        }
            }
            if (!free_spot) continue;
            for (int d = 0; d < 3; ++d) centres[3 * i + d] = c[d];
            cell[((size_t)ci[0] * nc[1] + ci[1]) * nc[2] + ci[2]].push_back(i);
            break;
        }
    }
    return ORC_OK;
}

}  // extern "C"
