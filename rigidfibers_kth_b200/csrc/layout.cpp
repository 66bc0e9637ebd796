// layout.cpp - seeded synthetic fiber layouts and geometry diagnostics.
//
// Replaces tools/gen.py of the reference (centres U[-2,2]^3, orientations
// from a cube then normalised, no minimum distance) with the generator the
// benchmark configurations specify: centres by rejection sampling with a
// minimum centre distance, uniform in a cube or isotropic Gaussian, and
// orientations uniform on the unit sphere (normalised N(0, I3) samples).
// The random stream is xoshiro256** seeded through splitmix64, so layouts are
// identical on every platform.
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "../../include/rigidfibers.h"

namespace {

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t z = seed;
        for (int i = 0; i < 4; ++i) {
            z += 0x9e3779b97f4a7c15ull;
            uint64_t x = z;
            x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
            x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
            s[i] = x ^ (x >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
    double normal() {
        // Box-Muller, one variate per call
        double u1 = uniform();
        while (u1 <= 0.0) u1 = uniform();
        const double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }
};

struct CellKey {
    int64_t operator()(int x, int y, int z) const {
        return ((int64_t)(x + 1048576) << 42) | ((int64_t)(y + 1048576) << 21) | (int64_t)(z + 1048576);
    }
};

}  // namespace

extern "C" rf_status rf_generate_layout(int32_t M, int32_t distribution, double box, double min_dist,
                                        uint64_t seed, double *positions, double *orientations) {
    if (M < 1 || !positions || !orientations || !(box > 0.0) || min_dist < 0.0 ||
        (distribution != 0 && distribution != 1))
        return RF_ERR_INVALID_ARG;
    if (distribution == 0) {
        // rough packing bound: spheres of diameter min_dist in the cube
        const double vol_needed = (double)M * (4.0 / 3.0) * M_PI * std::pow(0.5 * min_dist, 3.0);
        if (vol_needed > 0.5 * box * box * box) return RF_ERR_INVALID_ARG;
    }
    Rng rng(seed);
    const double cell = min_dist > 0.0 ? min_dist : 1.0;
    std::unordered_map<int64_t, std::vector<int>> grid;
    CellKey key;
    const double md2 = min_dist * min_dist;
    int placed = 0;
    int64_t attempts = 0;
    const int64_t max_attempts = (int64_t)M * 100000;
    while (placed < M) {
        if (++attempts > max_attempts) return RF_ERR_INVALID_ARG;
        double p[3];
        for (int a = 0; a < 3; ++a) p[a] = distribution == 0 ? box * rng.uniform() : box * rng.normal();
        const int cx = (int)std::floor(p[0] / cell), cy = (int)std::floor(p[1] / cell),
                  cz = (int)std::floor(p[2] / cell);
        bool ok = true;
        if (min_dist > 0.0) {
            for (int dx = -1; dx <= 1 && ok; ++dx)
                for (int dy = -1; dy <= 1 && ok; ++dy)
                    for (int dz = -1; dz <= 1 && ok; ++dz) {
                        auto it = grid.find(key(cx + dx, cy + dy, cz + dz));
                        if (it == grid.end()) continue;
                        for (int j : it->second) {
                            const double ddx = p[0] - positions[3 * j], ddy = p[1] - positions[3 * j + 1],
                                         ddz = p[2] - positions[3 * j + 2];
                            if (ddx * ddx + ddy * ddy + ddz * ddz < md2) {
                                ok = false;
                                break;
                            }
                        }
                    }
        }
        if (!ok) continue;
        for (int a = 0; a < 3; ++a) positions[3 * placed + a] = p[a];
        grid[key(cx, cy, cz)].push_back(placed);
        ++placed;
    }
    for (int i = 0; i < M; ++i) {
        double t[3], nrm = 0.0;
        do {
            nrm = 0.0;
            for (int a = 0; a < 3; ++a) {
                t[a] = rng.normal();
                nrm += t[a] * t[a];
            }
        } while (nrm < 1e-12);
        nrm = std::sqrt(nrm);
        for (int a = 0; a < 3; ++a) orientations[3 * i + a] = t[a] / nrm;
    }
    return RF_OK;
}

namespace {

// distance between segments p + s u and q + t v, s,t in [-1, 1] (unit u, v)
double segment_distance(const double *p, const double *u, const double *q, const double *v) {
    double w[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
    const double a = 1.0, b = u[0] * v[0] + u[1] * v[1] + u[2] * v[2], c = 1.0;
    const double d = u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
    const double e = v[0] * w[0] + v[1] * w[1] + v[2] * w[2];
    const double den = a * c - b * b;
    auto clamp = [](double x) { return x < -1.0 ? -1.0 : (x > 1.0 ? 1.0 : x); };
    double s, t;
    if (den > 1e-14) {
        s = clamp((b * e - c * d) / den);
    } else {
        s = 0.0;
    }
    t = clamp((b * s + e) / c);
    s = clamp((b * t - d) / a);
    double r[3];
    for (int k = 0; k < 3; ++k) r[k] = w[k] + s * u[k] - t * v[k];
    return std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

}  // namespace

extern "C" double rf_min_segment_distance(int32_t M, const double *positions, const double *orientations) {
    double best = INFINITY;
    for (int i = 0; i < M; ++i)
        for (int j = i + 1; j < M; ++j) {
            const double *p = positions + 3 * i, *q = positions + 3 * j;
            const double dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
            if (dx * dx + dy * dy + dz * dz > (2.0 + best) * (2.0 + best)) continue;
            const double dd = segment_distance(p, orientations + 3 * i, q, orientations + 3 * j);
            if (dd < best) best = dd;
        }
    return best;
}
