// Host-side input generators of the reference's GPU bench, built into
// libbrdc_inputs.so (plain g++, no CUDA).  They draw from the same <random>
// engines and distributions, seeded the same way and called in the same
// order, as gpu/bench/tridiag_dc_bench.cu:229-339, so a build against the
// same C++ standard library produces the same D and E bit for bit:
//
//   "bench"     D_i = n + i/4 + U(-1/2, 1/2), E_i = U(0.05, 0.95);
//               std::mt19937 seeded 1234 + (position of n in the bench's
//               size list)                               (:229-255)
//   "test"      an n x n matrix of U(-1, 1) drawn column by column; D is its
//               diagonal + n, E its first subdiagonal;
//               std::mt19937 seeded 1300 + n             (:307-333)
//   "normal"    D_i = N(0, 1), E_i = |N(0, 0.2)|         (:257-305, the
//   "uniform"   D_i = U(-1, 1), E_i = U(0.1, 0.3)         bench's paper
//   "toeplitz"  D_i = 2, E_i = 1/4                         modes; one
//   "clustered" D_i = 1 + 1e-12 (i - (n+1)/2),             std::mt19937_64
//               E_i = 1e-4 (1 + 0.1 cos(0.33 i)), i 1-based  per matrix)
//
// The paper modes' engine is seeded n * 0x9E3779B97F4A7C15 (mod 2^64)
// xor 0xD1B54A32D192ED03 for "normal", xor 0x94D049BB133111EB otherwise.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/brdc_inputs.h"

namespace {

void make_bench(int64_t n, uint32_t seed, double *D, double *E) {
    std::mt19937 eng(seed);
    std::uniform_real_distribution<double> jitter(-0.5, 0.5);
    std::uniform_real_distribution<double> coupling(0.05, 0.95);
    for (int64_t i = 0; i < n; ++i) {
        D[i] = static_cast<double>(n) + 0.25 * static_cast<double>(i) + jitter(eng);
    }
    for (int64_t i = 0; i + 1 < n; ++i) {
        E[i] = coupling(eng);
    }
}

void make_test(int64_t n, uint32_t seed, double *D, double *E) {
    std::mt19937 eng(seed);
    std::uniform_real_distribution<double> entry(-1.0, 1.0);
    // every entry of the dense matrix is drawn, column-major, and only the
    // diagonal and first subdiagonal are kept
    for (int64_t col = 0; col < n; ++col) {
        for (int64_t row = 0; row < n; ++row) {
            const double v = entry(eng);
            if (row == col) {
                D[col] = v + static_cast<double>(n);
            } else if (row == col + 1) {
                E[col] = v;
            }
        }
    }
}

enum PaperMode { kNormal, kUniform, kToeplitz, kClustered };

void make_paper(PaperMode mode, int64_t n, double *D, double *E) {
    const uint64_t base = static_cast<uint64_t>(n) * 0x9E3779B97F4A7C15ULL;
    const uint64_t salt = (mode == kNormal) ? 0xD1B54A32D192ED03ULL : 0x94D049BB133111EBULL;
    std::mt19937_64 eng(base ^ salt);
    std::normal_distribution<double> diag_n(0.0, 1.0);
    std::normal_distribution<double> off_n(0.0, 0.20);
    std::uniform_real_distribution<double> diag_u(-1.0, 1.0);
    std::uniform_real_distribution<double> off_u(0.10, 0.30);
    const double centre = 0.5 * (static_cast<double>(n) + 1.0);
    for (int64_t i = 0; i < n; ++i) {
        switch (mode) {
        case kNormal: D[i] = diag_n(eng); break;
        case kUniform: D[i] = diag_u(eng); break;
        case kToeplitz: D[i] = 2.0; break;
        case kClustered: D[i] = 1.0 + 1.0e-12 * (static_cast<double>(i + 1) - centre); break;
        }
    }
    for (int64_t i = 0; i + 1 < n; ++i) {
        switch (mode) {
        case kNormal: E[i] = std::abs(off_n(eng)); break;
        case kUniform: E[i] = off_u(eng); break;
        case kToeplitz: E[i] = 0.25; break;
        case kClustered: E[i] = 1.0e-4 * (1.0 + 0.1 * std::cos(0.33 * static_cast<double>(i + 1))); break;
        }
    }
}

} // namespace

extern "C" int brdc_input_generate(const char *mode, int64_t n, int64_t index,
                                   double *D, double *E) {
    if (mode == nullptr || D == nullptr || (n > 1 && E == nullptr)) {
        return BRDC_INPUT_BAD_ARGUMENT;
    }
    if (n < 1) {
        return BRDC_INPUT_BAD_ARGUMENT;
    }
    if (std::strcmp(mode, "bench") == 0) {
        make_bench(n, static_cast<uint32_t>(1234 + index), D, E);
    } else if (std::strcmp(mode, "test") == 0) {
        make_test(n, static_cast<uint32_t>(1300 + n), D, E);
    } else if (std::strcmp(mode, "normal") == 0) {
        make_paper(kNormal, n, D, E);
    } else if (std::strcmp(mode, "uniform") == 0) {
        make_paper(kUniform, n, D, E);
    } else if (std::strcmp(mode, "toeplitz") == 0) {
        make_paper(kToeplitz, n, D, E);
    } else if (std::strcmp(mode, "clustered") == 0) {
        make_paper(kClustered, n, D, E);
    } else {
        return BRDC_INPUT_UNKNOWN_MODE;
    }
    return BRDC_INPUT_OK;
}
