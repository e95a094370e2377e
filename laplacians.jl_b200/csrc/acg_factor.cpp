// Host-side randomized approximate Cholesky elimination (the `:deg` order).
//
// This produces the LDLinv factor that the GPU solve applies.  It restates
// the reference's elimination step by step so that, from the same seeded
// random stream, it makes the same choices:
//   LLmatp(a)              src/approxChol.jl:102-136   (linked columns)
//   flipIndex(a)           src/graphUtils.jl:49-55     (reverse edge index)
//   get_ll_col             src/approxChol.jl:354-385
//   compressCol!           src/approxChol.jl:415-449
//   approxChol(::LLmatp)   src/approxChol.jl:864-977
//   ApproxCholPQ & ops     src/approxChol.jl:2085-2239
// The two sorts inside compressCol! are Julia 1.8's `QuickSort` (Base.Sort:
// median-of-three pivot, insertion sort at <= 20 elements); equal keys are
// ordered by that algorithm, so it is restated here rather than replaced by
// std::sort.  `searchsortedfirst` (src/approxChol.jl:918) is a plain lower
// bound on a strictly increasing cumulative sum.
//
// Memory: edge records are struct-of-arrays indexed by CSC position, so the
// working set is 32 bytes per stored adjacency entry plus O(n).
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "acg_internal.h"
#include "acg_rng.h"

namespace acg {

namespace {

// Edge records of the linked-column matrix (LLp in src/approxCholTypes.jl:14-23).
struct LinkedCols {
  int64_t n = 0;
  std::vector<int64_t> row;   // 1-based vertex id of the row
  std::vector<double> val;    // weight; 0 marks a removed edge
  std::vector<int64_t> next;  // next record in the column; self terminates
  std::vector<int64_t> rev;   // record of the same edge in the other column
  std::vector<int64_t> head;  // head[v] (v 1-based) = first record of column v
  std::vector<int64_t> degs;  // initial degrees (1-based)
};

// Approximate priority queue on degrees (ApproxCholPQ; split = 1 for the :deg
// elimination, > 1 for the split/merge one, whose keys are split x degrees).
struct DegreeQueue {
  int64_t n = 0;
  int64_t split = 1;
  int64_t minlist = 1;
  int64_t nitems = 0;
  std::vector<int64_t> prev, next, key;  // indexed by 1-based vertex id; 0 = none
  std::vector<int64_t> lists;            // indexed 1..2*split*n+1

  int64_t key_map(int64_t x) const {
    const int64_t k = split * n, upper = 2 * split * n + 1;
    if (x <= k) return x;
    int64_t m = k + x / k;
    return m < upper ? m : upper;
  }

  void init(const std::vector<int64_t>& degs, int64_t nv, int64_t sp = 1) {
    n = nv;
    split = sp;
    prev.assign(n + 1, 0);
    next.assign(n + 1, 0);
    key.assign(n + 1, 0);
    lists.assign(2 * split * n + 2, 0);
    minlist = 1;
    nitems = n;
    for (int64_t i = 1; i <= n; ++i) {
      int64_t k = degs[i];
      if (k < 1 || k > 2 * split * n + 1) throw std::runtime_error("vertex degree out of queue range");
      int64_t h = lists[k];
      if (h > 0) {
        prev[i] = 0; next[i] = h; key[i] = k;
        prev[h] = i;  // next[h], key[h] unchanged
      } else {
        prev[i] = 0; next[i] = 0; key[i] = k;
      }
      lists[k] = i;
    }
  }

  int64_t pop() {
    if (nitems == 0) throw std::runtime_error("ApproxPQ is empty");
    while (lists[minlist] == 0) ++minlist;
    int64_t i = lists[minlist];
    int64_t nx = next[i];
    lists[minlist] = nx;
    if (nx > 0) prev[nx] = 0;
    --nitems;
    return i;
  }

  void move(int64_t i, int64_t newkey, int64_t oldlist, int64_t newlist) {
    int64_t pv = prev[i], nx = next[i];
    if (nx > 0) prev[nx] = pv;
    if (pv > 0) next[pv] = nx; else lists[oldlist] = nx;
    int64_t h = lists[newlist];
    if (h > 0) prev[h] = i;
    lists[newlist] = i;
    prev[i] = 0; next[i] = h; key[i] = newkey;
  }

  void dec(int64_t i) {
    int64_t oldlist = key_map(key[i]);
    int64_t newlist = key_map(key[i] - 1);
    if (newlist < 1) throw std::runtime_error("degree queue key underflow");
    if (newlist != oldlist) {
      move(i, key[i] - 1, oldlist, newlist);
      if (newlist < minlist) minlist = newlist;
    } else {
      key[i] -= 1;
    }
  }

  void inc(int64_t i) {
    int64_t oldlist = key_map(key[i]);
    int64_t newlist = key_map(key[i] + 1);
    if (newlist > 2 * split * n + 1) throw std::runtime_error("degree queue key overflow");
    if (newlist != oldlist) {
      move(i, key[i] + 1, oldlist, newlist);
    } else {
      key[i] += 1;
    }
  }
};

// Julia 1.8 Base.Sort QuickSort on v[lo..hi] (inclusive, 0-based) with a
// strict-weak "less" on the element handles.
template <class Less>
void julia_insertion_sort(int64_t* v, int64_t lo, int64_t hi, const Less& lt) {
  for (int64_t i = lo + 1; i <= hi; ++i) {
    int64_t j = i;
    int64_t x = v[i];
    while (j > lo) {
      if (lt(x, v[j - 1])) {
        v[j] = v[j - 1];
        --j;
        continue;
      }
      break;
    }
    v[j] = x;
  }
}

template <class Less>
int64_t julia_partition(int64_t* v, int64_t lo, int64_t hi, const Less& lt) {
  // selectpivot!: order v[mi] <= v[lo] <= v[hi]; the pivot ends in v[lo].
  int64_t mi = lo + ((hi - lo) >> 1);
  if (lt(v[lo], v[mi])) std::swap(v[mi], v[lo]);
  if (lt(v[hi], v[lo])) {
    if (lt(v[hi], v[mi])) {
      int64_t a = v[lo], b = v[mi], c = v[hi];
      v[hi] = a; v[lo] = b; v[mi] = c;
    } else {
      std::swap(v[hi], v[lo]);
    }
  }
  int64_t pivot = v[lo];
  int64_t i = lo, j = hi;
  while (true) {
    ++i; --j;
    while (lt(v[i], pivot)) ++i;
    while (lt(pivot, v[j])) --j;
    if (i >= j) break;
    std::swap(v[i], v[j]);
  }
  v[lo] = v[j];
  v[j] = pivot;
  return j;
}

template <class Less>
void julia_quicksort(int64_t* v, int64_t lo, int64_t hi, const Less& lt) {
  while (lo < hi) {
    if (hi - lo <= 20) {
      julia_insertion_sort(v, lo, hi, lt);
      return;
    }
    int64_t j = julia_partition(v, lo, hi, lt);
    if (j - lo < hi - j) {
      if (lo < j - 1) julia_quicksort(v, lo, j - 1, lt);
      lo = j + 1;
    } else {
      if (j + 1 < hi) julia_quicksort(v, j + 1, hi, lt);
      hi = j - 1;
    }
  }
}

void build_linked_cols(int64_t n, const int64_t* colptr, const int64_t* rowval,
                       const double* nzval, LinkedCols& ll) {
  const int64_t m = colptr[n] - colptr[0];
  ll.n = n;
  ll.row.resize(m);
  ll.val.resize(m);
  ll.next.resize(m);
  ll.rev.resize(m);
  ll.head.assign(n + 1, -1);
  ll.degs.assign(n + 1, 0);
  const int64_t base = colptr[0];
  for (int64_t i = 0; i < n; ++i) {
    int64_t p0 = colptr[i] - base, p1 = colptr[i + 1] - base;
    ll.degs[i + 1] = p1 - p0;
    if (p1 <= p0) throw std::runtime_error("vertex " + std::to_string(i + 1) + " has no edges");
    ll.row[p0] = rowval[p0];
    ll.val[p0] = nzval[p0];
    ll.next[p0] = p0;
    int64_t prevrec = p0;
    for (int64_t p = p0 + 1; p < p1; ++p) {
      ll.row[p] = rowval[p];
      ll.val[p] = nzval[p];
      ll.next[p] = prevrec;
      prevrec = p;
    }
    ll.head[i + 1] = prevrec;
  }
  // flipIndex: with rows sorted in every column and a symmetric pattern, the
  // records (row c, col r) are met in increasing c while scanning columns c.
  std::vector<int64_t> cursor(n, 0);
  for (int64_t c = 0; c < n; ++c) {
    for (int64_t p = colptr[c] - base; p < colptr[c + 1] - base; ++p) {
      int64_t r = rowval[p] - 1;
      int64_t q = colptr[r] - base + cursor[r]++;
      if (q >= colptr[r + 1] - base || rowval[q] != c + 1)
        throw std::runtime_error("adjacency matrix is not structurally symmetric with sorted rows");
      ll.rev[p] = q;
    }
  }
}

}  // namespace

void approx_chol_deg(int64_t n, const int64_t* colptr, const int64_t* rowval,
                     const double* nzval, JuliaRng* rng, HostFactor& out) {
  if (n < 2) throw std::runtime_error("approxChol needs at least 2 vertices");
  LinkedCols a;
  build_linked_cols(n, colptr, rowval, nzval, a);

  out.n = n;
  out.col.assign(n - 1, 0);
  out.colptr.assign(n, 0);
  out.rowval.clear();
  out.fval.clear();
  out.rowval.reserve((size_t)(a.row.size() * 0.6) + 16);
  out.fval.reserve((size_t)(a.row.size() * 0.6) + 16);
  out.d.assign(n, 0.0);

  DegreeQueue pq;
  pq.init(a.degs, n);

  std::vector<int64_t> colspace(n);
  std::vector<double> cumspace(n), vals(n);

  int64_t it = 1;  // 1-based elimination step, as in the reference
  int64_t ldli_row_ptr = 1;

  auto by_row = [&](int64_t x, int64_t y) { return a.row[x] < a.row[y]; };
  auto by_val = [&](int64_t x, int64_t y) { return a.val[x] < a.val[y]; };

  while (it < n) {
    int64_t i = pq.pop();
    out.col[it - 1] = i;
    out.colptr[it - 1] = ldli_row_ptr;
    ++it;

    // get_ll_col: walk the column, keep live records.
    int64_t len = 0;
    int64_t rec = a.head[i];
    while (true) {
      if (a.val[rec] > 0.0) {
        if (len >= (int64_t)colspace.size()) colspace.resize(2 * colspace.size() + 1);
        colspace[len++] = rec;
      }
      if (a.next[rec] == rec) break;
      rec = a.next[rec];
    }
    if (len == 0) throw std::runtime_error("eliminated vertex has no live edges (graph disconnected?)");

    // compressCol!: merge parallel edges, then order by weight.
    julia_quicksort(colspace.data(), 0, len - 1, by_row);
    int64_t ptr = -1;
    int64_t currow = 0;
    for (int64_t k = 0; k < len; ++k) {
      int64_t ck = colspace[k];
      if (a.row[ck] != currow) {
        currow = a.row[ck];
        ++ptr;
        colspace[ptr] = ck;
      } else {
        int64_t cp = colspace[ptr];
        a.val[cp] = a.val[cp] + a.val[ck];
        a.val[a.rev[ck]] = 0.0;
        pq.dec(currow);
      }
    }
    len = ptr + 1;
    julia_quicksort(colspace.data(), 0, len - 1, by_val);

    if ((int64_t)cumspace.size() < len) {
      cumspace.resize(len);
      vals.resize(len);
    }
    double csum = 0.0;
    for (int64_t k = 0; k < len; ++k) {
      vals[k] = a.val[colspace[k]];
      csum = csum + a.val[colspace[k]];
      cumspace[k] = csum;
    }
    double wdeg = csum;
    double colScale = 1.0;

    for (int64_t jo = 0; jo < len - 1; ++jo) {
      int64_t llr = colspace[jo];
      double w = vals[jo] * colScale;
      int64_t j = a.row[llr];
      int64_t revj = a.rev[llr];
      double f = w / wdeg;
      vals[jo] = 0.0;

      double r = julia_rand(rng) * (csum - cumspace[jo]) + cumspace[jo];
      // searchsortedfirst(cumspace, r, jo.., len): first index with cumspace >= r
      int64_t lo = -1, hi = len;  // over the full 1..len range like the reference
      while (lo < hi - 1) {
        int64_t mid = lo + ((hi - lo) >> 1);
        if (cumspace[mid] < r) lo = mid; else hi = mid;
      }
      int64_t koff = hi < len ? hi : len - 1;  // r can only exceed csum by rounding
      int64_t k = a.row[colspace[koff]];

      pq.inc(k);

      double newEdgeVal = f * (1.0 - f) * wdeg;

      // fix row k in col j
      a.row[revj] = k;
      a.val[revj] = newEdgeVal;
      a.rev[revj] = llr;

      // fix row j in col k
      int64_t khead = a.head[k];
      a.head[k] = llr;
      a.next[llr] = khead;
      a.rev[llr] = revj;
      a.val[llr] = newEdgeVal;
      a.row[llr] = j;

      colScale = colScale * (1.0 - f);
      double omf = 1.0 - f;
      wdeg = wdeg * (omf * omf);

      out.rowval.push_back(j);
      out.fval.push_back(f);
      ++ldli_row_ptr;
    }

    int64_t llr = colspace[len - 1];
    double w = vals[len - 1] * colScale;
    int64_t j = a.row[llr];
    int64_t revj = a.rev[llr];
    if (it < n) pq.dec(j);
    a.val[revj] = 0.0;
    out.rowval.push_back(j);
    out.fval.push_back(1.0);
    ++ldli_row_ptr;
    out.d[i - 1] = w;
  }
  out.colptr[it - 1] = ldli_row_ptr;
}

// Elimination in a fixed order: approxChol(::LLMatOrd) (src/approxChol.jl:758-862;
// the later of its two definitions, which is the one Julia keeps) on
// LLMatOrd(a) (src/approxChol.jl:203-229) or LLMatOrd(a, perm)
// (src/approxChol.jl:265-294), with the factor of a permuted order mapped back
// to the original vertex ids as approxchol_lapWdeg / approxchol_lapRandom do
// (src/approxChol.jl:1712-1713, 1770-1771).  perm (1-based, perm[k] = the
// vertex eliminated k-th) may be null: the given order 1..n.
void approx_chol_ord(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                     const int64_t* perm, JuliaRng* rng, HostFactor& out) {
  if (n < 2) throw std::runtime_error("approxChol needs at least 2 vertices");
  const int64_t base = colptr[0];
  const int64_t m = colptr[n] - base;
  std::vector<int64_t> invp(n + 1);
  if (perm) {
    std::vector<char> seen(n + 1, 0);
    for (int64_t k = 1; k <= n; ++k) {
      const int64_t v = perm[k - 1];
      if (v < 1 || v > n || seen[v]) throw std::runtime_error("perm is not a permutation of 1..n");
      seen[v] = 1;
      invp[v] = k;
    }
  } else {
    for (int64_t v = 1; v <= n; ++v) invp[v] = v;
  }
  // LLMatOrd: records 1..m (0 ends a column); column i holds the edges to j > i
  std::vector<int64_t> lrow(m + 1, 0), lnext(m + 1, 0);
  std::vector<double> lval(m + 1, 0.0);
  std::vector<int64_t> cols(n + 1, 0);
  int64_t rp = 1;
  for (int64_t i0 = 1; i0 <= (perm ? n : n - 1); ++i0) {
    const int64_t i = invp[i0];
    int64_t next = 0;
    for (int64_t ind = colptr[i0 - 1] - base; ind < colptr[i0] - base; ++ind) {
      const int64_t j = invp[rowval[ind]];
      if (i < j) {
        lrow[rp] = j;
        lnext[rp] = next;
        lval[rp] = nzval[ind];
        next = rp;
        ++rp;
      }
    }
    cols[i] = next;
  }

  out.n = n;
  out.col.assign(n - 1, 0);
  out.colptr.assign(n, 0);
  out.rowval.clear();
  out.fval.clear();
  out.d.assign(n, 0.0);
  std::vector<int64_t> crow, cptr, h, mrow, mptr;
  std::vector<double> cval, mval, cumspace;
  int64_t ldli_row_ptr = 1;
  for (int64_t i = 1; i <= n - 1; ++i) {
    out.col[i - 1] = i;
    out.colptr[i - 1] = ldli_row_ptr;
    // get_ll_col (src/approxChol.jl:387-410)
    int64_t len = 0;
    crow.clear();
    cptr.clear();
    cval.clear();
    for (int64_t q = cols[i]; q != 0; q = lnext[q]) {
      crow.push_back(lrow[q]);
      cptr.push_back(q);
      cval.push_back(lval[q]);
      ++len;
    }
    if (len == 0) throw std::runtime_error("eliminated vertex has no later neighbour (graph disconnected?)");
    // compressCol! on LLcol (src/approxChol.jl:451-492): QuickSort by row,
    // merge equal rows keeping the first record, QuickSort by value.
    h.resize(len);
    for (int64_t k = 0; k < len; ++k) h[k] = k;
    julia_quicksort(h.data(), 0, len - 1, [&](int64_t x, int64_t y) { return crow[x] < crow[y]; });
    mrow.clear();
    mptr.clear();
    mval.clear();
    int64_t currow = crow[h[0]], curptr = cptr[h[0]];
    double curval = cval[h[0]];
    for (int64_t k = 1; k < len; ++k) {
      const int64_t x = h[k];
      if (crow[x] != currow) {
        mrow.push_back(currow);
        mptr.push_back(curptr);
        mval.push_back(curval);
        currow = crow[x];
        curval = cval[x];
        curptr = cptr[x];
      } else {
        curval = curval + cval[x];
      }
    }
    mrow.push_back(currow);
    mptr.push_back(curptr);
    mval.push_back(curval);
    len = (int64_t)mrow.size();
    h.resize(len);
    for (int64_t k = 0; k < len; ++k) h[k] = k;
    julia_quicksort(h.data(), 0, len - 1, [&](int64_t x, int64_t y) { return mval[x] < mval[y]; });

    cumspace.resize(len);
    double csum = 0.0;
    for (int64_t k = 0; k < len; ++k) {
      csum = csum + mval[h[k]];
      cumspace[k] = csum;
    }
    double wdeg = csum;
    double colScale = 1.0;
    for (int64_t jo = 0; jo < len - 1; ++jo) {
      const int64_t c = h[jo];
      const double w = mval[c] * colScale;
      const int64_t j = mrow[c];
      const double f = w / wdeg;
      const double r = julia_rand(rng) * (csum - cumspace[jo]) + cumspace[jo];
      int64_t lo = -1, hi = len;  // searchsortedfirst over 1..len
      while (lo < hi - 1) {
        const int64_t mid = lo + ((hi - lo) >> 1);
        if (cumspace[mid] < r) lo = mid; else hi = mid;
      }
      const int64_t koff = hi < len ? hi : len - 1;  // r can only exceed csum by rounding
      const int64_t k = mrow[h[koff]];
      const double newEdgeVal = w * (1.0 - f);
      const int64_t q = mptr[c];
      if (j < k) {  // the new edge (j, k) goes into the lower column
        lrow[q] = k;
        lnext[q] = cols[j];
        lval[q] = newEdgeVal;
        cols[j] = q;
      } else {
        lrow[q] = j;
        lnext[q] = cols[k];
        lval[q] = newEdgeVal;
        cols[k] = q;
      }
      colScale = colScale * (1.0 - f);
      wdeg = wdeg - 2.0 * w + w * w / wdeg;
      out.rowval.push_back(j);
      out.fval.push_back(f);
      ++ldli_row_ptr;
    }
    const int64_t c = h[len - 1];
    out.rowval.push_back(mrow[c]);
    out.fval.push_back(1.0);
    ++ldli_row_ptr;
    out.d[i - 1] = mval[c] * colScale;
  }
  out.colptr[n - 1] = ldli_row_ptr;
  if (perm) {
    // LDLinv(p[col], colptr, p[rowval], fval, d[ip])
    for (auto& v : out.col) v = perm[v - 1];
    for (auto& v : out.rowval) v = perm[v - 1];
    std::vector<double> d2(n);
    for (int64_t v = 1; v <= n; ++v) d2[v - 1] = out.d[invp[v] - 1];
    out.d.swap(d2);
  }
}

// The split/merge elimination of approxchol_lap2: approxChol(a, split, merge)
// (src/approxChol.jl:979-1157) on LLmatp(a, split) (src/approxChol.jl:138-183),
// averaging parallel edges with compressAvgCol! (src/approxChol.jl:541-600).
// Every edge becomes `split` parallel records of weight w/split; record k of
// CSC entry p (0-based) is split*p + k, paired with record k of the entry's
// transpose.
// merge < 1 is approxChol(a, split) (src/approxChol.jl:1162-1322), which
// differs from the merge form only in averaging parallel edges with avgCol!
// (src/approxChol.jl:497-533) instead of compressAvgCol!: with no cap on the
// parallel edges compressAvgCol! keeps every record, divides by their count
// and sorts as avgCol! does, so merge < 1 runs as an unreachable cap.
void approx_chol_split(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                       int64_t split, int64_t merge, JuliaRng* rng, HostFactor& out) {
  if (n < 2) throw std::runtime_error("approxChol needs at least 2 vertices");
  if (split < 1) throw std::runtime_error("split must be at least 1");
  if (merge < 1) merge = INT64_MAX;
  const int64_t base = colptr[0];
  const int64_t nnz = colptr[n] - base;
  LinkedCols a;
  a.n = n;
  a.row.resize(split * nnz);
  a.val.resize(split * nnz);
  a.next.resize(split * nnz);
  a.rev.resize(split * nnz);
  a.head.assign(n + 1, -1);
  a.degs.assign(n + 1, 0);
  for (int64_t c = 0; c < n; ++c) {
    const int64_t p0 = colptr[c] - base, p1 = colptr[c + 1] - base;
    if (p1 <= p0) throw std::runtime_error("vertex " + std::to_string(c + 1) + " has no edges");
    a.degs[c + 1] = split * (p1 - p0);
    // the first entry: its last copy ends the column, the others chain to it
    int64_t prevrec = split * p0 + split - 1;
    a.row[prevrec] = rowval[p0];
    a.val[prevrec] = nzval[p0] / (double)split;
    a.next[prevrec] = prevrec;
    for (int64_t k = 0; k < split - 1; ++k) {
      const int64_t r = split * p0 + k;
      a.row[r] = rowval[p0];
      a.val[r] = nzval[p0] / (double)split;
      a.next[r] = prevrec;
      prevrec = r;
    }
    for (int64_t p = p0 + 1; p < p1; ++p) {
      for (int64_t k = 0; k < split; ++k) {
        const int64_t r = split * p + k;
        a.row[r] = rowval[p];
        a.val[r] = nzval[p] / (double)split;
        a.next[r] = prevrec;
        prevrec = r;
      }
    }
    a.head[c + 1] = prevrec;
  }
  {
    std::vector<int64_t> cursor(n, 0);
    for (int64_t c = 0; c < n; ++c) {
      for (int64_t p = colptr[c] - base; p < colptr[c + 1] - base; ++p) {
        const int64_t r = rowval[p] - 1;
        const int64_t q = colptr[r] - base + cursor[r]++;
        if (q >= colptr[r + 1] - base || rowval[q] != c + 1)
          throw std::runtime_error("adjacency matrix is not structurally symmetric with sorted rows");
        for (int64_t k = 0; k < split; ++k) a.rev[split * p + k] = split * q + k;
      }
    }
  }

  out.n = n;
  out.col.assign(n - 1, 0);
  out.colptr.assign(n, 0);
  out.rowval.clear();
  out.fval.clear();
  out.d.assign(n, 0.0);
  DegreeQueue pq;
  pq.init(a.degs, n, split);
  std::vector<int64_t> colspace(n);
  std::vector<double> vals(n), csr(n);
  int64_t it = 1;
  int64_t ldli_row_ptr = 1;
  auto by_row = [&](int64_t x, int64_t y) { return a.row[x] < a.row[y]; };
  auto by_val_row = [&](int64_t x, int64_t y) {
    return a.val[x] < a.val[y] || (a.val[x] == a.val[y] && a.row[x] < a.row[y]);
  };
  while (it < n) {
    const int64_t i = pq.pop();
    out.col[it - 1] = i;
    out.colptr[it - 1] = ldli_row_ptr;
    ++it;
    // get_ll_col
    int64_t len = 0;
    int64_t rec = a.head[i];
    while (true) {
      if (a.val[rec] > 0.0) {
        if (len >= (int64_t)colspace.size()) colspace.resize(2 * colspace.size() + 1);
        colspace[len++] = rec;
      }
      if (a.next[rec] == rec) break;
      rec = a.next[rec];
    }
    if (len == 0) throw std::runtime_error("eliminated vertex has no live edges (graph disconnected?)");
    // compressAvgCol!: QuickSort by row; average each run of parallel edges
    // (at most `merge` of them survive); QuickSort by (value, row).
    julia_quicksort(colspace.data(), 0, len - 1, by_row);
    int64_t ptr = 0;
    int64_t cur = 0, nxt = 0;
    while (nxt < len && a.row[colspace[cur]] == a.row[colspace[nxt]]) ++nxt;
    while (cur < len) {
      const int64_t num = nxt - cur;
      double mul_sum = 0.0;
      for (int64_t q = cur; q < nxt; ++q) mul_sum += a.val[colspace[q]];
      if (num <= merge) {
        const double nv = mul_sum / (double)num;
        for (int64_t q = cur; q < nxt; ++q) {
          const int64_t cr = colspace[q];
          a.val[cr] = nv;
          a.val[a.rev[cr]] = nv;
          colspace[ptr++] = cr;
        }
      } else {
        const double nv = mul_sum / (double)merge;
        for (int64_t q = cur; q < cur + merge; ++q) {
          const int64_t cr = colspace[q];
          a.val[cr] = nv;
          a.val[a.rev[cr]] = nv;
          colspace[ptr++] = cr;
        }
        const int64_t currow = a.row[colspace[cur]];
        for (int64_t q = cur + merge; q < nxt; ++q) {
          a.val[a.rev[colspace[q]]] = 0.0;
          pq.dec(currow);
        }
      }
      cur = nxt;
      while (nxt < len && a.row[colspace[cur]] == a.row[colspace[nxt]]) ++nxt;
    }
    len = ptr;
    julia_quicksort(colspace.data(), 0, len - 1, by_val_row);

    if ((int64_t)vals.size() < len) {
      vals.resize(len);
      csr.resize(len);
    }
    double csum = 0.0;
    for (int64_t q = 0; q < len; ++q) {
      csum = csum + a.val[colspace[q]];
      vals[q] = a.val[colspace[q]];
    }
    double csum_rev = 0.0;  // csr[q] = sum of the values from q to the end
    for (int64_t q = len - 1; q >= 0; --q) {
      csum_rev += a.val[colspace[q]];
      csr[q] = csum_rev;
    }
    double wdeg = csum;
    double colScale = 1.0;
    int64_t next_edge = 0;  // the first entry that is not a parallel copy of the current neighbour
    double final_d = 0.0;
    for (int64_t jo = 0; jo < len - 1; ++jo) {
      const bool is_new = jo == next_edge;
      while (next_edge < len && a.row[colspace[jo]] == a.row[colspace[next_edge]]) ++next_edge;
      if (next_edge == len) {
        // only copies of the last neighbour remain: no self loop is created
        for (int64_t q = jo; q < len - 1; ++q) {
          const int64_t cr = colspace[q];
          final_d += vals[q] * colScale;
          if (it < n) pq.dec(a.row[cr]);
          a.val[a.rev[cr]] = 0.0;
        }
        break;
      }
      const int64_t llr = colspace[jo];
      const double w = vals[jo] * colScale;
      const int64_t j = a.row[llr];
      const int64_t revj = a.rev[llr];
      double f = w / wdeg;
      vals[jo] = 0.0;
      const double r = julia_rand(rng) * csr[next_edge];
      // searchsortedlast on the non-increasing csr: the last q with csr[q] >= r
      int64_t lo = -1, hi = len;
      while (lo < hi - 1) {
        const int64_t mid = lo + ((hi - lo) >> 1);
        if (csr[mid] < r) hi = mid; else lo = mid;
      }
      const int64_t koff = lo < 0 ? 0 : lo;
      const int64_t k = a.row[colspace[koff]];
      pq.inc(k);
      const double newEdgeVal = a.val[llr] * csr[next_edge] / csum;
      a.row[revj] = k;
      a.val[revj] = newEdgeVal;
      a.rev[revj] = llr;
      const int64_t khead = a.head[k];
      a.head[k] = llr;
      a.next[llr] = khead;
      a.rev[llr] = revj;
      a.val[llr] = newEdgeVal;
      a.row[llr] = j;
      if (is_new) {
        out.rowval.push_back(j);
        out.fval.push_back(f);
        ++ldli_row_ptr;
      } else {
        out.fval.back() = out.fval.back() + f;
      }
      if (jo == next_edge - 1) {  // the last copy of this neighbour
        f = out.fval.back();
        colScale = colScale * (1.0 - f);
        const double omf = 1.0 - f;
        wdeg = wdeg * (omf * omf);
      }
    }
    const int64_t llr = colspace[len - 1];
    final_d += vals[len - 1] * colScale;
    const int64_t j = a.row[llr];
    if (it < n) pq.dec(j);
    a.val[a.rev[llr]] = 0.0;
    out.rowval.push_back(j);
    out.fval.push_back(1.0);
    ++ldli_row_ptr;
    out.d[i - 1] = final_d;
  }
  out.colptr[it - 1] = ldli_row_ptr;
}

}  // namespace acg
