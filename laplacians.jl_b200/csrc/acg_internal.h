// Internal host-side types shared by the C-ABI translation units.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "acg_rng.h"

namespace acg {

// The LDLinv factor as the reference stores it (src/approxCholTypes.jl:73-79):
// 1-based vertex ids, col[ii] = vertex eliminated at step ii (n-1 of them),
// colptr (n entries, colptr[n-1] = F+1), rowval/fval (F), d (n, by vertex).
struct HostFactor {
  int64_t n = 0;
  std::vector<int64_t> col, colptr, rowval;
  std::vector<double> fval, d;
};

void approx_chol_deg(int64_t n, const int64_t* colptr, const int64_t* rowval,
                     const double* nzval, JuliaRng* rng, HostFactor& out);
// Elimination in a fixed order (perm: 1-based, null = 1..n); see acg_factor.cpp.
void approx_chol_ord(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                     const int64_t* perm, JuliaRng* rng, HostFactor& out);
// The split/merge elimination of approxchol_lap2; see acg_factor.cpp.
void approx_chol_split(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                       int64_t split, int64_t merge, JuliaRng* rng, HostFactor& out);

// Opt-in elimination in rounds of independent low-degree vertices on `threads`
// host threads, with its own keyed random numbers; see acg_factor_par.cpp.
void approx_chol_parallel(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                          uint64_t seed, int threads, HostFactor& out, int64_t* rounds);

// Thread-local error text returned by acg_last_error().
void set_last_error(const std::string& msg);

}  // namespace acg
