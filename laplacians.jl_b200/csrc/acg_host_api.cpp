// C-ABI entry points that run on the host only: the Julia-compatible random
// stream and the approximate Cholesky elimination.  See include/acgpu.h.
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "../../include/acgpu.h"
#include "acg_internal.h"

struct acg_factor {
  acg::HostFactor f;
};

namespace acg {
namespace {
thread_local std::string g_last_error;
}
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace acg

extern "C" {

const char* acg_last_error(void) { return acg::g_last_error.c_str(); }

int acg_rng_seed(uint64_t seed, uint64_t state[4]) {
  if (!state) {
    acg::set_last_error("acg_rng_seed: null state");
    return ACG_ERR_INVALID;
  }
  acg::JuliaRng r;
  acg::julia_seed(&r, seed);
  std::memcpy(state, r.s, sizeof(r.s));
  return ACG_OK;
}

int acg_rng_rand(uint64_t state[4], double* out, int64_t count) {
  if (!state || (!out && count > 0) || count < 0) {
    acg::set_last_error("acg_rng_rand: bad arguments");
    return ACG_ERR_INVALID;
  }
  acg::JuliaRng r;
  std::memcpy(r.s, state, sizeof(r.s));
  for (int64_t k = 0; k < count; ++k) out[k] = acg::julia_rand(&r);
  std::memcpy(state, r.s, sizeof(r.s));
  return ACG_OK;
}

int acg_sha256(const uint8_t* data, int64_t len, uint8_t out[32]) {
  if ((!data && len > 0) || len < 0 || !out) {
    acg::set_last_error("acg_sha256: bad arguments");
    return ACG_ERR_INVALID;
  }
  acg::sha256(data, (size_t)len, out);
  return ACG_OK;
}

namespace {

// Shared by acg_approxchol (:deg) and acg_approxchol_ordered (a fixed order).
// mode 0: :deg; 1: a fixed order (perm, null = given); 2: split/merge
int approxchol_entry(const char* name, int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                     const int64_t* perm, int mode, int64_t split, int64_t merge, uint64_t rng_state[4],
                     acg_factor** out) {
  if (!out || !colptr || !rowval || !nzval || !rng_state || n < 2) {
    acg::set_last_error(std::string(name) + ": bad arguments (need n >= 2 and non-null arrays)");
    return ACG_ERR_INVALID;
  }
  *out = nullptr;
  const int64_t base = colptr[0];
  if (base != 0 && base != 1) {
    acg::set_last_error(std::string(name) + ": colptr[0] must be 0 or 1");
    return ACG_ERR_INVALID;
  }
  try {
    const int64_t m = colptr[n] - base;
    for (int64_t p = 0; p < m; ++p) {
      if (!(nzval[p] >= 0.0)) {
        acg::set_last_error("Adjacency matrix can not have negative edge weights");
        return ACG_ERR_INVALID;
      }
    }
    // The elimination works on 1-based rows like the reference; shift 0-based input.
    const int64_t* rv = rowval;
    std::vector<int64_t> shifted;
    if (base == 0) {
      shifted.resize(m);
      for (int64_t p = 0; p < m; ++p) shifted[p] = rowval[p] + 1;
      rv = shifted.data();
    }
    for (int64_t p = 0; p < m; ++p) {
      if (rv[p] < 1 || rv[p] > n) {
        acg::set_last_error(std::string(name) + ": row index out of range");
        return ACG_ERR_INVALID;
      }
    }
    acg::JuliaRng r;
    std::memcpy(r.s, rng_state, sizeof(r.s));
    auto* fac = new acg_factor();
    try {
      if (mode == 1) acg::approx_chol_ord(n, colptr, rv, nzval, perm, &r, fac->f);
      else if (mode == 2) acg::approx_chol_split(n, colptr, rv, nzval, split, merge, &r, fac->f);
      else acg::approx_chol_deg(n, colptr, rv, nzval, &r, fac->f);
    } catch (...) {
      delete fac;
      throw;
    }
    std::memcpy(rng_state, r.s, sizeof(r.s));
    *out = fac;
    return ACG_OK;
  } catch (const std::bad_alloc&) {
    acg::set_last_error(std::string(name) + ": host out of memory");
    return ACG_ERR_NOMEM;
  } catch (const std::exception& e) {
    acg::set_last_error(std::string(name) + ": " + e.what());
    return ACG_ERR_INVALID;
  }
}

}  // namespace

int acg_approxchol(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                   uint64_t rng_state[4], acg_factor** out) {
  return approxchol_entry("acg_approxchol", n, colptr, rowval, nzval, nullptr, 0, 1, 1, rng_state, out);
}

int acg_approxchol_ordered(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                           const int64_t* perm, uint64_t rng_state[4], acg_factor** out) {
  return approxchol_entry("acg_approxchol_ordered", n, colptr, rowval, nzval, perm, 1, 1, 1, rng_state, out);
}

int acg_approxchol_parallel(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                            uint64_t seed, int threads, int64_t* rounds, acg_factor** out) {
  if (!out || !colptr || !rowval || !nzval || n < 2) {
    acg::set_last_error("acg_approxchol_parallel: bad arguments (need n >= 2 and non-null arrays)");
    return ACG_ERR_INVALID;
  }
  *out = nullptr;
  if (colptr[0] != 0 && colptr[0] != 1) {
    acg::set_last_error("acg_approxchol_parallel: colptr[0] must be 0 or 1");
    return ACG_ERR_INVALID;
  }
  auto* fac = new acg_factor();
  try {
    acg::approx_chol_parallel(n, colptr, rowval, nzval, seed, threads, fac->f, rounds);
  } catch (const std::bad_alloc&) {
    delete fac;
    acg::set_last_error("acg_approxchol_parallel: host out of memory");
    return ACG_ERR_NOMEM;
  } catch (const std::exception& e) {
    delete fac;
    acg::set_last_error(std::string("acg_approxchol_parallel: ") + e.what());
    return ACG_ERR_INVALID;
  }
  *out = fac;
  return ACG_OK;
}

int acg_approxchol_split(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval, int64_t split,
                         int64_t merge, uint64_t rng_state[4], acg_factor** out) {
  if (split < 1 || split > 64) {
    acg::set_last_error("acg_approxchol_split: need 1 <= split <= 64");
    return ACG_ERR_INVALID;
  }
  return approxchol_entry("acg_approxchol_split", n, colptr, rowval, nzval, nullptr, 2, split, merge, rng_state, out);
}

int acg_factor_dims(const acg_factor* f, int64_t* n, int64_t* nnz) {
  if (!f || !n || !nnz) {
    acg::set_last_error("acg_factor_dims: null argument");
    return ACG_ERR_INVALID;
  }
  *n = f->f.n;
  *nnz = (int64_t)f->f.fval.size();
  return ACG_OK;
}

int acg_factor_export(const acg_factor* f, int64_t* col, int64_t* colptr, int64_t* rowval,
                      double* fval, double* d) {
  if (!f || !col || !colptr || !rowval || !fval || !d) {
    acg::set_last_error("acg_factor_export: null argument");
    return ACG_ERR_INVALID;
  }
  const acg::HostFactor& h = f->f;
  std::memcpy(col, h.col.data(), sizeof(int64_t) * h.col.size());
  std::memcpy(colptr, h.colptr.data(), sizeof(int64_t) * h.colptr.size());
  std::memcpy(rowval, h.rowval.data(), sizeof(int64_t) * h.rowval.size());
  std::memcpy(fval, h.fval.data(), sizeof(double) * h.fval.size());
  std::memcpy(d, h.d.data(), sizeof(double) * h.d.size());
  return ACG_OK;
}

void acg_factor_free(acg_factor* f) { delete f; }

// ---- binary LDLinv file ------------------------------------------------------
//
// Little-endian: the 8 bytes "ACGLDLI1", int64 n, int64 F, int64 index base
// (always 1), then col[n-1], colptr[n], rowval[F] as int64 and fval[F], d[n]
// as float64: the LDLinv fields of src/approxCholTypes.jl:73-79 as Julia
// stores them.

int acg_ldlinv_save(const char* path, int64_t n, const int64_t* col, const int64_t* colptr, const int64_t* rowval,
                    const double* fval, const double* d, int64_t nnz) {
  if (!path || n < 1 || nnz < 0 || !colptr || !d || (n > 1 && !col) || (nnz > 0 && (!rowval || !fval))) {
    acg::set_last_error("acg_ldlinv_save: bad arguments");
    return ACG_ERR_INVALID;
  }
  FILE* fh = std::fopen(path, "wb");
  if (!fh) {
    acg::set_last_error(std::string("acg_ldlinv_save: cannot open ") + path);
    return ACG_ERR_INVALID;
  }
  const int64_t head[3] = {n, nnz, 1};
  bool ok = std::fwrite("ACGLDLI1", 1, 8, fh) == 8 && std::fwrite(head, sizeof(int64_t), 3, fh) == 3;
  ok = ok && std::fwrite(col, sizeof(int64_t), (size_t)(n - 1), fh) == (size_t)(n - 1);
  ok = ok && std::fwrite(colptr, sizeof(int64_t), (size_t)n, fh) == (size_t)n;
  ok = ok && std::fwrite(rowval, sizeof(int64_t), (size_t)nnz, fh) == (size_t)nnz;
  ok = ok && std::fwrite(fval, sizeof(double), (size_t)nnz, fh) == (size_t)nnz;
  ok = ok && std::fwrite(d, sizeof(double), (size_t)n, fh) == (size_t)n;
  ok = (std::fclose(fh) == 0) && ok;
  if (!ok) {
    acg::set_last_error(std::string("acg_ldlinv_save: write failed: ") + path);
    return ACG_ERR_INVALID;
  }
  return ACG_OK;
}

int acg_ldlinv_load(const char* path, acg_factor** out) {
  if (!path || !out) {
    acg::set_last_error("acg_ldlinv_load: null argument");
    return ACG_ERR_INVALID;
  }
  *out = nullptr;
  FILE* fh = std::fopen(path, "rb");
  if (!fh) {
    acg::set_last_error(std::string("acg_ldlinv_load: cannot open ") + path);
    return ACG_ERR_INVALID;
  }
  auto fail = [&](const char* why) {
    std::fclose(fh);
    acg::set_last_error(std::string("acg_ldlinv_load: ") + why + ": " + path);
    return ACG_ERR_INVALID;
  };
  char magic[8];
  int64_t head[3];
  if (std::fread(magic, 1, 8, fh) != 8 || std::memcmp(magic, "ACGLDLI1", 8) != 0) return fail("not an LDLinv file");
  if (std::fread(head, sizeof(int64_t), 3, fh) != 3) return fail("truncated header");
  const int64_t n = head[0], nnz = head[1];
  if (n < 1 || nnz < 0 || head[2] != 1) return fail("bad header");
  // the payload must be exactly the size the header announces
  std::fseek(fh, 0, SEEK_END);
  const long long bytes = std::ftell(fh);
  const long long want = 32 + 8LL * ((n - 1) + n + nnz + nnz + n);
  if (bytes != want) return fail("file size does not match its header");
  std::fseek(fh, 32, SEEK_SET);
  try {
    auto* f = new acg_factor();
    acg::HostFactor& h = f->f;
    h.n = n;
    h.col.resize((size_t)(n - 1));
    h.colptr.resize((size_t)n);
    h.rowval.resize((size_t)nnz);
    h.fval.resize((size_t)nnz);
    h.d.resize((size_t)n);
    bool ok = std::fread(h.col.data(), sizeof(int64_t), h.col.size(), fh) == h.col.size();
    ok = ok && std::fread(h.colptr.data(), sizeof(int64_t), h.colptr.size(), fh) == h.colptr.size();
    ok = ok && std::fread(h.rowval.data(), sizeof(int64_t), h.rowval.size(), fh) == h.rowval.size();
    ok = ok && std::fread(h.fval.data(), sizeof(double), h.fval.size(), fh) == h.fval.size();
    ok = ok && std::fread(h.d.data(), sizeof(double), h.d.size(), fh) == h.d.size();
    // structure: colptr runs from 1 to F+1 without decreasing, ids in [1, n]
    ok = ok && h.colptr[0] == 1 && h.colptr[(size_t)(n - 1)] == nnz + 1;
    for (size_t i = 1; ok && i < h.colptr.size(); ++i) ok = h.colptr[i] >= h.colptr[i - 1];
    for (size_t i = 0; ok && i < h.col.size(); ++i) ok = h.col[i] >= 1 && h.col[i] <= n;
    for (size_t i = 0; ok && i < h.rowval.size(); ++i) ok = h.rowval[i] >= 1 && h.rowval[i] <= n;
    if (!ok) {
      delete f;
      return fail("malformed factor");
    }
    std::fclose(fh);
    *out = f;
    return ACG_OK;
  } catch (const std::bad_alloc&) {
    std::fclose(fh);
    acg::set_last_error("acg_ldlinv_load: host out of memory");
    return ACG_ERR_NOMEM;
  }
}

}  // extern "C"
