// Opt-in parallel approximate Cholesky elimination on the host.
//
// The reference's elimination (src/approxChol.jl:864-977) is sequential: one
// vertex at a time, in approximate minimum-degree order, each choice drawn
// from the global rand() stream.  This variant eliminates in rounds.  Each
// round takes the live vertices of degree at most max(2, the median live
// degree) whose degree is a local minimum (a vertex is taken when its (degree,
// pseudo-random priority) is below every live neighbour's: an independent set
// of low-degree vertices) and eliminates the whole set at once on several
// threads.  No two vertices of a round are
// adjacent, so their eliminations read disjoint columns; the new edges they
// sample are merged into the graph after the round.  The last 4,096 vertices
// (the nearly dense end of the elimination), or a remainder in which a round
// takes under 1/64 of the vertices, are eliminated one at a time in minimum-
// degree order.
//
// Each single elimination is the reference's step: merge parallel edges,
// order the column by weight, and for every entry but the last sample a
// neighbour further along the column with probability proportional to its
// weight, join the two with weight f (1 - f) wdeg, and scale the rest
// (src/approxChol.jl:888-966).  The random numbers come from a counter-based
// generator keyed by (seed, vertex, entry) instead of Julia's stream, so the
// factor is NOT the reference's (a different, equally valid sample); it does
// not depend on the number of threads.
//
// What it buys: the factor's dependency DAG, up to the sequential remainder,
// is at most as deep as the number of rounds (a vertex depends only on
// vertices of earlier rounds), and the rounds run on all host cores.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "acg_internal.h"

namespace acg {

namespace {

uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// uniform in [0, 1) from (seed, a, b): 53 random bits
double u01(uint64_t seed, uint64_t a, uint64_t b) {
  const uint64_t h = mix64(seed ^ mix64(a * 0x100000001b3ull ^ mix64(b + 0x632be59bd9b4e019ull)));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

// body(t, begin, end) on `threads` threads over [0, count) in contiguous chunks
// (serially below `serial_below`).
template <class F>
void parallel_chunks(int threads, int64_t count, int64_t serial_below, const F& body) {
  if (threads <= 1 || count < serial_below) {
    body(0, 0, count);
    return;
  }
  std::vector<std::thread> pool;
  const int64_t chunk = (count + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const int64_t b = t * chunk, e = std::min<int64_t>(count, b + chunk);
    if (b >= e) break;
    pool.emplace_back([&, t, b, e]() { body(t, b, e); });
  }
  for (auto& th : pool) th.join();
}

template <class F>
void parallel_for(int threads, int64_t count, const F& body) {
  parallel_chunks(threads, count, 2048, [&](int, int64_t b, int64_t e) { body(b, e); });
}

struct Edge {
  int32_t to;
  double w;
};

// Merge parallel edges, drop edges to eliminated vertices; entries by neighbour
// id.  Parallel edges are summed in order of weight, so the result does not
// depend on the order in which the edges were appended.
void compress(std::vector<Edge>& adj, const std::vector<uint8_t>& dead) {
  size_t k = 0;
  for (const Edge& e : adj)
    if (!dead[e.to] && e.w > 0.0) adj[k++] = e;
  adj.resize(k);
  std::sort(adj.begin(), adj.end(),
            [](const Edge& x, const Edge& y) { return x.to < y.to || (x.to == y.to && x.w < y.w); });
  size_t p = 0;
  for (size_t i = 0; i < adj.size(); ++i) {
    if (p > 0 && adj[p - 1].to == adj[i].to) adj[p - 1].w += adj[i].w;
    else adj[p++] = adj[i];
  }
  adj.resize(p);
}

struct Column {
  std::vector<int32_t> rows;
  std::vector<double> fvals;
  double d = 0.0;
  std::vector<std::pair<int32_t, int32_t>> new_edges;  // (j, k)
  std::vector<double> new_w;
};

// The reference's elimination of one vertex on its compressed column
// (src/approxChol.jl:888-966), sampling with the keyed generator.
void eliminate(int32_t u, const std::vector<Edge>& col_in, uint64_t seed, Column& out) {
  std::vector<Edge> col(col_in);
  std::sort(col.begin(), col.end(), [](const Edge& x, const Edge& y) {
    return x.w < y.w || (x.w == y.w && x.to < y.to);
  });
  const int64_t len = (int64_t)col.size();
  std::vector<double> cum(len);
  double csum = 0.0;
  for (int64_t i = 0; i < len; ++i) {
    csum += col[i].w;
    cum[i] = csum;
  }
  double wdeg = csum, colScale = 1.0;
  out.rows.clear();
  out.fvals.clear();
  out.new_edges.clear();
  out.new_w.clear();
  for (int64_t jo = 0; jo + 1 < len; ++jo) {
    const int32_t j = col[jo].to;
    const double w = col[jo].w * colScale;
    const double f = w / wdeg;
    const double r = u01(seed, (uint64_t)u, (uint64_t)jo) * (csum - cum[jo]) + cum[jo];
    int64_t koff = std::lower_bound(cum.begin() + jo + 1, cum.end(), r) - cum.begin();
    if (koff >= len) koff = len - 1;
    const int32_t k = col[koff].to;
    out.new_edges.emplace_back(j, k);
    out.new_w.push_back(f * (1.0 - f) * wdeg);
    colScale *= (1.0 - f);
    wdeg *= (1.0 - f) * (1.0 - f);
    out.rows.push_back(j);
    out.fvals.push_back(f);
  }
  out.rows.push_back(col[len - 1].to);
  out.fvals.push_back(1.0);
  out.d = col[len - 1].w * colScale;
}

// Buckets of vertices by count (doubly linked lists), counts above `top`
// sharing the last bucket: O(1) moves, the minimum found by a cursor that only
// moves up between decrements.
struct CountBuckets {
  int64_t top;
  std::vector<int32_t> head, prev, next;
  std::vector<int64_t> key;
  int64_t cur = 0;
  CountBuckets(int32_t n, int64_t top_) : top(top_), head(top_ + 1, -1), prev(n, -1), next(n, -1), key(n, -1) {}
  int64_t slot(int64_t c) const { return c < top ? c : top; }
  void insert(int32_t v, int64_t c) {
    key[v] = c;
    const int64_t b = slot(c);
    prev[v] = -1;
    next[v] = head[b];
    if (head[b] >= 0) prev[head[b]] = v;
    head[b] = v;
    if (b < cur) cur = b;
  }
  void remove(int32_t v) {
    const int64_t b = slot(key[v]);
    if (prev[v] >= 0) next[prev[v]] = next[v];
    else head[b] = next[v];
    if (next[v] >= 0) prev[next[v]] = prev[v];
  }
  void change(int32_t v, int64_t c) {
    remove(v);
    insert(v, c);
  }
  // the vertex with the smallest count (the first of its bucket; in the top
  // bucket, the smallest key there)
  int32_t pop_min() {
    while (cur <= top && head[cur] < 0) ++cur;
    int32_t v = head[cur];
    if (cur == top)
      for (int32_t w = head[cur]; w >= 0; w = next[w])
        if (key[w] < key[v]) v = w;
    remove(v);
    return v;
  }
};

// Finish the elimination one vertex at a time in minimum-degree order.  Each
// live vertex keeps a count of its live column entries (parallel edges
// counted apart, as the reference's degree queue counts them): minus one for
// each eliminated neighbour, plus one for each sampled edge.  Leaves the last
// vertex as the root.
void sequential_tail(std::vector<int32_t>& alive, std::vector<std::vector<Edge>>& adj, std::vector<uint8_t>& dead,
                     std::vector<uint8_t>& dirty, uint64_t seed, HostFactor& out) {
  CountBuckets q((int32_t)adj.size(), 4096);
  for (int32_t v : alive) {
    compress(adj[v], dead);
    dirty[v] = 0;
    q.insert(v, (int64_t)adj[v].size());
  }
  size_t remaining = alive.size();
  Column col;
  while (remaining > 1) {
    const int32_t u = q.pop_min();
    compress(adj[u], dead);
    if (adj[u].empty()) throw std::runtime_error("eliminated vertex has no live edges (graph disconnected?)");
    eliminate(u, adj[u], seed, col);
    dead[u] = 1;
    --remaining;
    out.col.push_back(u + 1);
    out.colptr.push_back((int64_t)out.rowval.size() + 1);
    for (size_t i = 0; i < col.rows.size(); ++i) {
      out.rowval.push_back(col.rows[i] + 1);
      out.fval.push_back(col.fvals[i]);
    }
    out.d[u] = col.d;
    for (const Edge& ed : adj[u]) q.change(ed.to, q.key[ed.to] - 1);  // the neighbours lose u
    for (size_t i = 0; i < col.new_edges.size(); ++i) {
      const int32_t j = col.new_edges[i].first, k = col.new_edges[i].second;
      adj[j].push_back({k, col.new_w[i]});
      adj[k].push_back({j, col.new_w[i]});
      q.change(j, q.key[j] + 1);
      q.change(k, q.key[k] + 1);
    }
    std::vector<Edge>().swap(adj[u]);
  }
  int32_t root = -1;
  for (int32_t v : alive)
    if (!dead[v]) root = v;
  alive.assign(1, root);
}

}  // namespace

void approx_chol_parallel(int64_t n64, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                          uint64_t seed, int threads, HostFactor& out, int64_t* rounds_out) {
  if (n64 < 2 || n64 >= (int64_t)INT32_MAX) throw std::runtime_error("parallel elimination needs 2 <= n < 2^31");
  const int32_t n = (int32_t)n64;
  if (threads < 1) threads = 1;
  const int64_t base = colptr[0];
  std::vector<std::vector<Edge>> adj(n);
  for (int32_t c = 0; c < n; ++c) {
    const int64_t p0 = colptr[c] - base, p1 = colptr[c + 1] - base;
    if (p1 <= p0) throw std::runtime_error("vertex " + std::to_string(c + 1) + " has no edges");
    adj[c].reserve(p1 - p0);
    for (int64_t p = p0; p < p1; ++p) {
      const int64_t r = rowval[p] - base;
      if (r < 0 || r >= n) throw std::runtime_error("row index out of range");
      if (!(nzval[p] >= 0.0) || std::isinf(nzval[p]))
        throw std::runtime_error("Adjacency matrix can not have negative edge weights");
      if (r != c && nzval[p] > 0.0) adj[c].push_back({(int32_t)r, nzval[p]});
    }
  }
  std::vector<uint8_t> dead(n, 0), dirty(n, 1);
  std::vector<int32_t> alive(n);
  for (int32_t v = 0; v < n; ++v) alive[v] = v;
  out.n = n;
  out.col.clear();
  out.colptr.clear();
  out.rowval.clear();
  out.fval.clear();
  out.d.assign(n, 0.0);
  int64_t rounds = 0;
  std::vector<Column> cols;
  std::vector<int32_t> chosen;
  while (alive.size() > 1) {
    // compress the columns that changed
    parallel_for(threads, (int64_t)alive.size(), [&](int64_t b, int64_t e) {
      for (int64_t i = b; i < e; ++i) {
        const int32_t v = alive[i];
        if (dirty[v]) {
          compress(adj[v], dead);
          dirty[v] = 0;
        }
      }
    });
    // candidates: live degree at most max(2, the median live degree), so that
    // leaves and degree-2 vertices (whose eliminations are exact) go first, as
    // in the minimum-degree order
    int64_t maxdeg = 0;
    for (int32_t v : alive) maxdeg = std::max<int64_t>(maxdeg, (int64_t)adj[v].size());
    std::vector<int64_t> hist(maxdeg + 2, 0);
    for (int32_t v : alive) hist[adj[v].size()]++;
    size_t cap = 0;
    for (int64_t acc = 0; cap <= (size_t)maxdeg; ++cap) {
      acc += hist[cap];
      if (2 * acc >= (int64_t)alive.size()) break;
    }
    cap = std::max<size_t>(cap, 2);
    // an independent set: the candidates whose (degree, priority) is below every
    // live neighbour's, i.e. local minima of the degree
    auto prio = [&](int32_t v) { return mix64(seed ^ mix64(((uint64_t)rounds << 32) ^ (uint64_t)v)); };
    std::vector<uint8_t> pick(alive.size(), 0);
    parallel_for(threads, (int64_t)alive.size(), [&](int64_t b, int64_t e) {
      for (int64_t i = b; i < e; ++i) {
        const int32_t v = alive[i];
        const size_t dv = adj[v].size();
        if (dv == 0 || dv > cap) continue;  // isolated vertices are reported below
        const uint64_t pv = prio(v);
        bool win = true;
        for (const Edge& ed : adj[v]) {
          const size_t du = adj[ed.to].size();
          if (du < dv || (du == dv && prio(ed.to) < pv) || (du == dv && prio(ed.to) == pv && ed.to < v)) {
            win = false;
            break;
          }
        }
        pick[i] = win;
      }
    });
    for (int32_t v : alive)
      if (adj[v].empty()) throw std::runtime_error("eliminated vertex has no live edges (graph disconnected?)");
    chosen.clear();
    for (size_t i = 0; i < alive.size(); ++i)
      if (pick[i]) chosen.push_back(alive[i]);
    // a round never takes the last live vertex (the root)
    if (chosen.size() == alive.size()) chosen.pop_back();
    // the last few thousand vertices (the nearly dense end of the elimination,
    // which the solver's dense tail replaces anyway), or a remainder in which a
    // round takes under 1/64 of the vertices (a round costs a pass over every
    // live column, a single elimination only its own): one vertex at a time
    if (alive.size() <= 4096 || chosen.size() * 64 < alive.size()) {
      sequential_tail(alive, adj, dead, dirty, seed, out);
      ++rounds;
      break;
    }
    // eliminate the set
    cols.resize(chosen.size());
    parallel_for(threads, (int64_t)chosen.size(), [&](int64_t b, int64_t e) {
      for (int64_t i = b; i < e; ++i) eliminate(chosen[i], adj[chosen[i]], seed, cols[i]);
    });
    // record the columns in the order of the set
    for (size_t i = 0; i < chosen.size(); ++i) {
      const int32_t u = chosen[i];
      dead[u] = 1;
      out.col.push_back(u + 1);
      out.colptr.push_back((int64_t)out.rowval.size() + 1);
      for (size_t q = 0; q < cols[i].rows.size(); ++q) {
        out.rowval.push_back(cols[i].rows[q] + 1);
        out.fval.push_back(cols[i].fvals[q]);
      }
      out.d[u] = cols[i].d;
    }
    // merge the sampled edges: each thread sorts its eliminations' records into
    // buckets by owner thread of the target vertex (target % T), then each
    // thread appends the records of the vertices it owns; a record with
    // neighbour -1 only marks its target (a neighbour of an eliminated vertex)
    const int T = (int)std::min<int64_t>(threads, std::max<int64_t>(1, (int64_t)chosen.size() / 256));
    std::vector<std::vector<std::vector<Edge>>> bucket_to(T, std::vector<std::vector<Edge>>(T));
    std::vector<std::vector<std::vector<int32_t>>> bucket_at(T, std::vector<std::vector<int32_t>>(T));
    parallel_chunks(T, (int64_t)chosen.size(), 1, [&](int t, int64_t b, int64_t e) {
      auto& bt = bucket_to[t];
      auto& ba = bucket_at[t];
      for (int64_t i = b; i < e; ++i) {
        for (const Edge& ed : adj[chosen[i]]) {
          ba[ed.to % T].push_back(ed.to);
          bt[ed.to % T].push_back({-1, 0.0});
        }
        for (size_t q = 0; q < cols[i].new_edges.size(); ++q) {
          const int32_t j = cols[i].new_edges[q].first, k = cols[i].new_edges[q].second;
          const double w = cols[i].new_w[q];
          ba[j % T].push_back(j);
          bt[j % T].push_back({k, w});
          ba[k % T].push_back(k);
          bt[k % T].push_back({j, w});
        }
      }
    });
    parallel_chunks(T, T, 1, [&](int, int64_t b, int64_t e) {
      for (int64_t owner = b; owner < e; ++owner)
        for (int t = 0; t < T; ++t) {
          const auto& at = bucket_at[t][owner];
          const auto& to = bucket_to[t][owner];
          for (size_t q = 0; q < at.size(); ++q) {
            dirty[at[q]] = 1;
            if (to[q].to >= 0) adj[at[q]].push_back(to[q]);
          }
        }
    });
    for (int32_t u : chosen) std::vector<Edge>().swap(adj[u]);
    size_t k = 0;
    for (int32_t v : alive)
      if (!dead[v]) alive[k++] = v;
    alive.resize(k);
    ++rounds;
  }
  out.colptr.push_back((int64_t)out.rowval.size() + 1);
  if (rounds_out) *rounds_out = rounds;
}

}  // namespace acg
