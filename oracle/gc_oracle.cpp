// CPU oracle for the tiled push-relabel graph cut.  TEST INFRASTRUCTURE ONLY: the parity
// tests, the smoke check and the CPU-baseline leg of the benchmark use it to check results;
// nothing in the product links or loads it.
//
// Three parts, all int32/int64 arithmetic:
//   * orc_maxflow_bk   - an exact max-flow written from the published Boykov-Kolmogorov
//                        augmenting-path method (Boykov & Kolmogorov, "An Experimental
//                        Comparison of Min-Cut/Max-Flow Algorithms for Energy Minimization
//                        in Vision", IEEE TPAMI 26(9), 2004).  Independent of the reference
//                        schedule and of the CUDA solver.
//   * orc_canonical    - the canonical cut of a final residual state: the pixels reachable
//                        from pixels with excess > 0 over residual n-link edges (the minimal
//                        source set), and the flow value sum(max(t,0)) - sum(max(e,0)).
//   * orc_ref_tiled    - an int32 restatement of the reference's own schedule: GraphCut.cut
//                        (GraphCut.pyx:348-418) driving the graphcut.cl kernels (wave pushes
//                        in four directions, add_border, Jacobi relabel, tiled BFS global
//                        relabel, completion check) over IncrementalTileList stamps.  Each
//                        kernel below cites the reference lines it follows.  It is the CPU
//                        baseline (OpenMP over tiles) and a second independent solver.
//
// Parity status: the flow value of a graph is unique, and so is its canonical cut (the
// minimal source set), so orc_maxflow_bk pins both for any correct solver.  Both parts are
// pinned to the reference's own kernels: graphcut.cl, compiled unchanged for the host and
// run under the reference's host loop (refcl_host.c), gives orc_maxflow_bk's flow and cut
// on the golden graphs (tests/golden/refcl_*.npz, among them the reference's own test
// input), and orc_ref_tiled ends in the kernels' cut after the kernels' push iterations
// and relabel passes on every graph tried, including one where both stop short of the
// maximum flow.  The primitives (scan, compaction, tile lists) are pinned against the
// reference's own test vectors.
//
// Plane layout: row-major int32 [H][W]; up/down/left/right hold the residual capacity of
// the edge from the pixel to that neighbour; excess is the signed t-link (positive:
// source capacity, negative: sink capacity).  Capacities that leave the image are ignored.

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum Dir { UP = 0, DOWN = 1, LEFT = 2, RIGHT = 3 };
inline int rev(int d) { return d ^ 1; }

struct Grid {
  int W, H;
  long long N;
  inline bool has(long long i, int d) const {
    int x = (int)(i % W), y = (int)(i / W);
    switch (d) {
      case UP: return y > 0;
      case DOWN: return y < H - 1;
      case LEFT: return x > 0;
      default: return x < W - 1;
    }
  }
  inline long long nb(long long i, int d) const {
    switch (d) {
      case UP: return i - W;
      case DOWN: return i + W;
      case LEFT: return i - 1;
      default: return i + 1;
    }
  }
};

// ------------------------------------------------------------------------------------
// Canonical cut and flow value of a residual state.
// ------------------------------------------------------------------------------------
void canonical_labels(const Grid& g, const int32_t* const rc[4], const int64_t* exc,
                      uint8_t* labels) {
  std::vector<long long> q;
  q.reserve(1024);
  for (long long i = 0; i < g.N; ++i) {
    labels[i] = exc[i] > 0 ? 1 : 0;
    if (labels[i]) q.push_back(i);
  }
  for (size_t k = 0; k < q.size(); ++k) {
    long long u = q[k];
    for (int d = 0; d < 4; ++d) {
      if (!g.has(u, d) || rc[d][u] <= 0) continue;
      long long v = g.nb(u, d);
      if (!labels[v]) { labels[v] = 1; q.push_back(v); }
    }
  }
}

int64_t flow_value(long long n, const int32_t* t0, const int64_t* e) {
  int64_t s = 0;
  for (long long i = 0; i < n; ++i) s += std::max<int64_t>(t0[i], 0) - std::max<int64_t>(e[i], 0);
  return s;
}

// ------------------------------------------------------------------------------------
// Boykov-Kolmogorov max-flow (TPAMI 2004): two search trees S and T grown from the
// terminals, augmentation along the S-T path found, adoption of orphans.
// ------------------------------------------------------------------------------------
struct BK {
  Grid g;
  std::vector<int32_t> rc[4];
  std::vector<int64_t> tr;      // terminal residual: >0 from source, <0 to sink
  std::vector<uint8_t> tree;    // 0 free, 1 S, 2 T
  std::vector<int8_t> parent;   // 0..3 direction to parent, 4 terminal, 5 orphan/none
  std::vector<int32_t> ts, dist;
  std::vector<uint8_t> inq;
  std::deque<long long> active, orphans;
  int32_t TIME = 0;
  int64_t flow = 0;

  static constexpr int8_t TERM = 4, NONE = 5;

  void init(int W, int H, const int32_t* const caps[4], const int32_t* exc) {
    g = Grid{W, H, (long long)W * H};
    for (int d = 0; d < 4; ++d) {
      rc[d].assign(g.N, 0);
      for (long long i = 0; i < g.N; ++i) rc[d][i] = g.has(i, d) ? caps[d][i] : 0;
    }
    tr.resize(g.N);
    tree.assign(g.N, 0);
    parent.assign(g.N, NONE);
    ts.assign(g.N, 0);
    dist.assign(g.N, 0);
    inq.assign(g.N, 0);
    for (long long i = 0; i < g.N; ++i) {
      tr[i] = exc[i];
      if (tr[i] > 0) tree[i] = 1;
      else if (tr[i] < 0) tree[i] = 2;
      if (tree[i]) { parent[i] = TERM; dist[i] = 1; push_active(i); }
    }
  }
  void push_active(long long i) {
    if (!inq[i]) { inq[i] = 1; active.push_back(i); }
  }
  // residual capacity of the tree edge "parent -> child" (S) or "child -> parent" (T)
  inline int32_t tree_cap_in(long long child, int8_t pd, uint8_t t) const {
    long long p = g.nb(child, pd);
    return t == 1 ? rc[rev(pd)][p] : rc[pd][child];
  }

  void augment(long long a, long long b, int dab) {
    // a in S, b in T, edge a -> b in direction dab
    int64_t f = rc[dab][a];
    long long x = a;
    while (parent[x] != TERM) { int8_t pd = parent[x]; long long y = g.nb(x, pd); f = std::min<int64_t>(f, rc[rev(pd)][y]); x = y; }
    f = std::min<int64_t>(f, tr[x]);
    x = b;
    while (parent[x] != TERM) { int8_t pd = parent[x]; f = std::min<int64_t>(f, rc[pd][x]); x = g.nb(x, pd); }
    f = std::min<int64_t>(f, -tr[x]);

    rc[dab][a] -= (int32_t)f;
    rc[rev(dab)][b] += (int32_t)f;
    x = a;
    while (parent[x] != TERM) {
      int8_t pd = parent[x]; long long y = g.nb(x, pd);
      rc[rev(pd)][y] -= (int32_t)f; rc[pd][x] += (int32_t)f;
      if (rc[rev(pd)][y] == 0) { parent[x] = NONE; orphans.push_front(x); }
      x = y;
    }
    tr[x] -= f;
    if (tr[x] == 0) { parent[x] = NONE; orphans.push_front(x); }
    x = b;
    while (parent[x] != TERM) {
      int8_t pd = parent[x]; long long y = g.nb(x, pd);
      rc[pd][x] -= (int32_t)f; rc[rev(pd)][y] += (int32_t)f;
      if (rc[pd][x] == 0) { parent[x] = NONE; orphans.push_front(x); }
      x = y;
    }
    tr[x] += f;
    if (tr[x] == 0) { parent[x] = NONE; orphans.push_front(x); }
    flow += f;
  }

  void adopt(long long x) {
    uint8_t t = tree[x];
    int best = -1;
    int32_t dmin = INT32_MAX;
    for (int d = 0; d < 4; ++d) {
      if (!g.has(x, d)) continue;
      long long y = g.nb(x, d);
      if (tree[y] != t) continue;
      int32_t cap = t == 1 ? rc[rev(d)][y] : rc[d][x];
      if (cap <= 0) continue;
      // origin check: walk to a terminal; ts == TIME marks nodes verified this round
      long long j = y;
      int32_t dd = 0;
      bool ok = false;
      while (true) {
        if (ts[j] == TIME) { dd += dist[j]; ok = true; break; }
        int8_t pj = parent[j];
        dd++;
        if (pj == TERM) { ts[j] = TIME; dist[j] = 1; ok = true; break; }
        if (pj == NONE) break;
        j = g.nb(j, pj);
      }
      if (!ok) continue;
      if (dd < dmin) { dmin = dd; best = d; }
      // stamp the verified path
      j = y;
      int32_t dj = dd;
      while (ts[j] != TIME) { ts[j] = TIME; dist[j] = dj--; j = g.nb(j, parent[j]); }
    }
    if (best >= 0) {
      parent[x] = (int8_t)best; ts[x] = TIME; dist[x] = dmin + 1;
      return;
    }
    // no parent found: x becomes free
    for (int d = 0; d < 4; ++d) {
      if (!g.has(x, d)) continue;
      long long y = g.nb(x, d);
      if (tree[y] != t) continue;
      int32_t cap = t == 1 ? rc[rev(d)][y] : rc[d][x];
      if (cap > 0) push_active(y);
      int8_t py = parent[y];
      if (py >= 0 && py < 4 && g.nb(y, py) == x) { parent[y] = NONE; orphans.push_back(y); }
    }
    tree[x] = 0;
  }

  void run() {
    while (!active.empty()) {
      long long p = active.front();
      if (tree[p] == 0) { active.pop_front(); inq[p] = 0; continue; }
      long long a = -1, b = -1;
      int dab = -1;
      for (int d = 0; d < 4 && a < 0; ++d) {
        if (!g.has(p, d)) continue;
        long long q = g.nb(p, d);
        int32_t cap = tree[p] == 1 ? rc[d][p] : rc[rev(d)][q];
        if (cap <= 0) continue;
        if (tree[q] == 0) {
          tree[q] = tree[p]; parent[q] = (int8_t)rev(d); ts[q] = ts[p]; dist[q] = dist[p] + 1;
          push_active(q);
        } else if (tree[q] != tree[p]) {
          if (tree[p] == 1) { a = p; b = q; dab = d; } else { a = q; b = p; dab = rev(d); }
        } else if (ts[q] <= ts[p] && dist[q] > dist[p]) {
          parent[q] = (int8_t)rev(d); ts[q] = ts[p]; dist[q] = dist[p] + 1;
        }
      }
      if (a < 0) { active.pop_front(); inq[p] = 0; continue; }
      ++TIME;
      augment(a, b, dab);
      while (!orphans.empty()) { long long o = orphans.front(); orphans.pop_front(); adopt(o); }
    }
  }
};

// ------------------------------------------------------------------------------------
// Restatement of the reference schedule (GraphCut.pyx + graphcut.cl), int32.
// ------------------------------------------------------------------------------------
enum Op { OP_EQUAL = 0, OP_GT = 1, OP_LT = 2, OP_GTE = 3, OP_LTE = 4 };

inline bool apply_op(int op, int32_t v, int32_t operand) {
  switch (op) {
    case OP_EQUAL: return v == operand;
    case OP_GT: return v > operand;
    case OP_LT: return v < operand;
    case OP_GTE: return v >= operand;
    default: return v <= operand;
  }
}

// IncrementalTileList (IncrementalTileList.pyx:37-189; incremental_tile_list.cl:26-154).
struct TileList {
  std::vector<int32_t> tiles;  // per-tile iteration stamps (d_tiles)
  std::vector<int32_t> list;   // compacted tile ids (d_list)
  int32_t iteration = 0;
  void reset(int n) { tiles.assign(n, -1); iteration = 0; list.clear(); }   // :178-189
  int32_t increment() { return ++iteration; }                                  // :114-117
  void build(int op, int32_t operand) {                                        // :119-136
    list.clear();                 // flag (.cl:40-64) + StreamCompact.compact: the compaction
    for (int i = 0; i < (int)tiles.size(); ++i)   // is an exclusive scan of the flags then a
      if (apply_op(op, tiles[i], operand)) list.push_back(i);   // scatter (streamcompact.cl)
  }
  void build() { build(OP_EQUAL, iteration); }
  void incorporate(const std::vector<int32_t>& t2, int op1, int32_t a1, int op2, int32_t a2,
                   bool logical_and) {                                         // :138-155
    for (size_t i = 0; i < tiles.size(); ++i) {
      bool f1 = apply_op(op1, tiles[i], a1), f2 = apply_op(op2, t2[i], a2);
      if (logical_and ? (f1 && f2) : (f1 || f2)) tiles[i] = iteration;
    }
  }
  int length() const { return (int)list.size(); }
};

struct TiledRef {
  static constexpr int TILE = 32, WAVE = 8, NWAVE = 4;
  int W, H, TW, TH, NT;
  int32_t MAXH;
  std::vector<int32_t> exc, hgt, hgt2, cap[4], src[4], border;
  std::vector<uint8_t> loaded;
  TileList load, bfs, edges, brd;
  long long pushes = 0, relabels = 0, bfs_rounds = 0, iterations = 0;

  inline int32_t& C(int d, int x, int y) { return cap[d][(long long)y * W + x]; }
  inline int32_t& E(int x, int y) { return exc[(long long)y * W + x]; }
  inline int32_t& Hh(int x, int y) { return hgt[(long long)y * W + x]; }

  void setup(int W_, int H_, const int32_t* const caps[4], const int32_t* e) {
    W = W_; H = H_; TW = W / TILE; TH = H / TILE; NT = TW * TH;
    MAXH = W * H;                                                   // GraphCut.pyx:88
    long long N = (long long)W * H;
    exc.assign(e, e + N);
    for (int d = 0; d < 4; ++d) {
      src[d].assign(caps[d], caps[d] + N);
      cap[d].assign(N, 0);
    }
    for (int x = 0; x < W; ++x) { src[UP][x] = 0; src[DOWN][(long long)(H - 1) * W + x] = 0; }
    for (int y = 0; y < H; ++y) { src[LEFT][(long long)y * W] = 0; src[RIGHT][(long long)y * W + W - 1] = 0; }
    hgt.assign(N, 0);     // reference buffers are uninitialised; zero here (see file header)
    hgt2.assign(N, 0);
    border.assign((long long)TH * W, 0);
    loaded.assign(NT, 0);
    load.reset(NT); bfs.reset(NT); edges.reset(NT); brd.reset(NT);
  }

  // init_gc (graphcut.cl:63-112): zero the capacity planes, stamp tiles with excess >= 0.
  void init_gc(int32_t it) {
    for (int d = 0; d < 4; ++d) std::fill(cap[d].begin(), cap[d].end(), 0);
#pragma omp parallel for schedule(static)
    for (int t = 0; t < NT; ++t) {
      int tx = t % TW, ty = t / TW;
      bool any = false;
      for (int y = ty * TILE; y < (ty + 1) * TILE && !any; ++y)
        for (int x = tx * TILE; x < (tx + 1) * TILE; ++x)
          if (E(x, y) >= 0) { any = true; break; }
      if (any) load.tiles[t] = it;
    }
  }

  // Capacity upload in place of load_tiles (graphcut.cl:1033-1132): the tile's uploaded
  // capacities are added to its residual planes, which until now hold only the reverse
  // flow that neighbours pushed into it.  (load_tiles assigns the last row's down and the
  // last column's right capacity, graphcut.cl:1104,1130, which drops that reverse flow;
  // the restatement adds.)
  void load_tiles(const std::vector<int32_t>& list) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < (int)list.size(); ++k) {
      int t = list[k];
      if (loaded[t]) continue;
      loaded[t] = 1;
      int tx = t % TW, ty = t / TW;
      for (int y = ty * TILE; y < (ty + 1) * TILE; ++y)
        for (int x = tx * TILE; x < (tx + 1) * TILE; ++x) {
          long long i = (long long)y * W + x;
          for (int d = 0; d < 4; ++d) cap[d][i] += src[d][i];
        }
    }
  }

  // push_down (graphcut.cl:403-470) / push_up (:472-536): per column and per 8-pixel wave,
  // flow carried pixel to pixel; the wave's end flow goes to the next wave's first pixel
  // after all waves finished, or, for the tile's last wave, to the border buffer.
  void push_vertical(bool down, int32_t it) {
    const auto& L = load.list;
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < (int)L.size(); ++k) {
      int t = L[k], tx = t % TW, ty = t / TW;
      bool flag = false;
      int32_t over[TILE];
      for (int lx = 0; lx < TILE; ++lx) {
        int x = tx * TILE + lx;
        int32_t carry[NWAVE];
        for (int ly = 0; ly < NWAVE; ++ly) {
          int32_t flow = 0;
          int y0 = ty * TILE + ly * WAVE;
          for (int s = 0; s < WAVE; ++s) {
            int y = down ? y0 + s : y0 + WAVE - 1 - s;
            int yn = down ? y + 1 : y - 1;
            int32_t ef = E(x, y) + flow;
            bool inside = down ? (yn < H) : (yn >= 0);
            int32_t h = Hh(x, y);
            int32_t hn = inside ? Hh(x, yn) : MAXH;
            int dcap = down ? DOWN : UP;
            if (inside && ef > 0 && h < MAXH && h == hn + 1) flow = std::min(ef, C(dcap, x, y));
            else flow = 0;
            C(dcap, x, y) -= flow;
            E(x, y) = ef - flow;
            if (inside) C(rev(dcap), x, yn) += flow;
          }
          carry[ly] = flow;
        }
        // after the barrier: carries into the neighbouring wave, overspill to the border
        for (int ly = 0; ly < NWAVE; ++ly) {
          if (down) {
            if (ly != NWAVE - 1) E(x, ty * TILE + (ly + 1) * WAVE) += carry[ly];
            else { over[lx] = carry[ly]; if (carry[ly] > 0) flag = true; }
          } else {
            if (ly != 0) E(x, ty * TILE + ly * WAVE - 1) += carry[ly];
            else { over[lx] = carry[ly]; if (carry[ly] > 0) flag = true; }
          }
        }
      }
      if (flag) {
        int ny = down ? ty + 1 : ty - 1;
        for (int lx = 0; lx < TILE; ++lx) border[(long long)ny * W + tx * TILE + lx] = over[lx];
        brd.tiles[ny * TW + tx] = it;
      }
    }
  }

  // push_right (graphcut.cl:282-401) / push_left (:158-279): the same waves along rows
  // (the reference stores left/right capacities tile-transposed; the logical edge order is
  // restated here on a row-major layout).
  void push_horizontal(bool right, int32_t it) {
    const auto& L = load.list;
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < (int)L.size(); ++k) {
      int t = L[k], tx = t % TW, ty = t / TW;
      bool flag = false;
      int32_t over[TILE];
      for (int lx = 0; lx < TILE; ++lx) {
        int y = ty * TILE + lx;
        int32_t carry[NWAVE];
        for (int ly = 0; ly < NWAVE; ++ly) {
          int32_t flow = 0;
          int x0 = tx * TILE + ly * WAVE;
          for (int s = 0; s < WAVE; ++s) {
            int x = right ? x0 + s : x0 + WAVE - 1 - s;
            int xn = right ? x + 1 : x - 1;
            int32_t ef = E(x, y) + flow;
            bool inside = right ? (xn < W) : (xn >= 0);
            int32_t h = Hh(x, y);
            int32_t hn = inside ? Hh(xn, y) : MAXH;
            int dcap = right ? RIGHT : LEFT;
            if (inside && ef > 0 && h < MAXH && h == hn + 1) flow = std::min(ef, C(dcap, x, y));
            else flow = 0;
            C(dcap, x, y) -= flow;
            E(x, y) = ef - flow;
            if (inside) C(rev(dcap), xn, y) += flow;
          }
          carry[ly] = flow;
        }
        for (int ly = 0; ly < NWAVE; ++ly) {
          if (right) {
            if (ly != NWAVE - 1) E(tx * TILE + (ly + 1) * WAVE, y) += carry[ly];
            else { over[lx] = carry[ly]; if (carry[ly] > 0) flag = true; }
          } else {
            if (ly != 0) E(tx * TILE + ly * WAVE - 1, y) += carry[ly];
            else { over[lx] = carry[ly]; if (carry[ly] > 0) flag = true; }
          }
        }
      }
      if (flag) {
        int nx = right ? tx + 1 : tx - 1;
        for (int lx = 0; lx < TILE; ++lx) border[(long long)ty * W + nx * TILE + lx] = over[lx];
        brd.tiles[ty * TW + nx] = it;
      }
    }
  }

  // add_border (graphcut.cl:114-156): the overspill of the neighbouring tile enters this
  // tile's first row (0), last row (1), first column (2) or last column (3).
  void add_border(int direction) {
    const auto& L = brd.list;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < (int)L.size(); ++k) {
      int t = L[k], tx = t % TW, ty = t / TW;
      for (int lx = 0; lx < TILE; ++lx) {
        int32_t b = border[(long long)ty * W + tx * TILE + lx];
        int x, y;
        switch (direction) {
          case 0: x = tx * TILE + lx; y = ty * TILE; break;
          case 1: x = tx * TILE + lx; y = (ty + 1) * TILE - 1; break;
          case 2: x = tx * TILE; y = ty * TILE + lx; break;
          default: x = (tx + 1) * TILE - 1; y = ty * TILE + lx; break;
        }
        E(x, y) += b;
      }
    }
  }

  // GraphCut.push (GraphCut.pyx:242-323).
  void push() {
    push_vertical(true, brd.increment());
    brd.build(); if (brd.length()) add_border(0);
    push_vertical(false, brd.increment());
    brd.build(); if (brd.length()) add_border(1);
    push_horizontal(true, brd.increment());
    brd.build(); if (brd.length()) add_border(2);
    push_horizontal(false, brd.increment());
    brd.build(); if (brd.length()) add_border(3);
  }

  // relabel (graphcut.cl:538-577) + the buffer swap (GraphCut.pyx:224-240): Jacobi over
  // the whole image, active pixels take min(h_neighbour + 1) over residual edges.
  void relabel() {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x) {
        long long i = (long long)y * W + x;
        int32_t h = hgt[i], nh = h;
        if (exc[i] > 0 && h < MAXH) {
          nh = MAXH;
          if (y < H - 1 && cap[DOWN][i] > 0) nh = std::min(nh, hgt[i + W] + 1);
          if (y > 0 && cap[UP][i] > 0) nh = std::min(nh, hgt[i - W] + 1);
          if (x < W - 1 && cap[RIGHT][i] > 0) nh = std::min(nh, hgt[i + 1] + 1);
          if (x > 0 && cap[LEFT][i] > 0) nh = std::min(nh, hgt[i - 1] + 1);
        }
        hgt2[i] = nh;
      }
    hgt.swap(hgt2);
  }

  // init_bfs (graphcut.cl:582-802): distance seeds (0 where excess < 0, else MAX) for the
  // loaded tiles, distance 1 for tile-edge pixels whose neighbour across the edge is a sink
  // pixel they can push to, and the stamp of tiles that need the in-tile BFS.  The left
  // case tests tx (the reference tests ty, graphcut.cl:746).
  void init_bfs(int32_t it) {
    const auto& L = load.list;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < (int)L.size(); ++k) {
      int t = L[k], tx = t % TW, ty = t / TW;
      bool has_neg = false, has_nonneg = false, seeded = false;
      for (int y = ty * TILE; y < (ty + 1) * TILE; ++y)
        for (int x = tx * TILE; x < (tx + 1) * TILE; ++x) {
          if (E(x, y) >= 0) { Hh(x, y) = MAXH; has_nonneg = true; }
          else { Hh(x, y) = 0; has_neg = true; }
        }
      for (int l = 0; l < TILE; ++l) {
        int x, y;
        x = tx * TILE + l; y = ty * TILE;
        if (ty > 0 && C(UP, x, y) > 0 && E(x, y) >= 0 && E(x, y - 1) < 0) { Hh(x, y) = 1; seeded = true; }
        y = (ty + 1) * TILE - 1;
        if (ty < TH - 1 && C(DOWN, x, y) > 0 && E(x, y) >= 0 && E(x, y + 1) < 0) { Hh(x, y) = 1; seeded = true; }
        x = (tx + 1) * TILE - 1; y = ty * TILE + l;
        if (tx < TW - 1 && C(RIGHT, x, y) > 0 && E(x, y) >= 0 && E(x + 1, y) < 0) { Hh(x, y) = 1; seeded = true; }
        x = tx * TILE;
        if (tx > 0 && C(LEFT, x, y) > 0 && E(x, y) >= 0 && E(x - 1, y) < 0) { Hh(x, y) = 1; seeded = true; }
      }
      if (seeded || (has_neg && has_nonneg)) bfs.tiles[t] = it;
    }
  }

  // bfs_intratile (graphcut.cl:871-1016): in-tile min-relaxation d(u) = min(d(u), d(v)+1)
  // over residual u -> v with MAX padding, up to 30 rounds.  One pass per tile (the
  // reference launches two work-groups per tile, GraphCut.pyx:157).  A tile that hits the
  // round cap while still changing is stamped for another round so the BFS stays exact.
  bool intratile(int32_t it_edges, int32_t it_bfs_next) {
    bool capped = false;
    const auto& L = bfs.list;
#pragma omp parallel for schedule(dynamic, 2)
    for (int k = 0; k < (int)L.size(); ++k) {
      int t = L[k], tx = t % TW, ty = t / TW;
      int x0 = tx * TILE, y0 = ty * TILE;
      int rounds = 0;
      bool changed = true;
      while (changed && rounds < 30) {
        changed = false;
        for (int lx = 0; lx < TILE; ++lx)
          for (int ly = 0; ly < NWAVE; ++ly) {
            int x = x0 + lx;
            for (int s = 0; s < WAVE; ++s) {          // up pass (top to bottom)
              int y = y0 + ly * WAVE + s;
              if (y > y0 && C(UP, x, y) > 0 && Hh(x, y - 1) + 1 < Hh(x, y)) { Hh(x, y) = Hh(x, y - 1) + 1; changed = true; }
            }
            for (int s = WAVE - 1; s >= 0; --s) {     // down pass (bottom to top)
              int y = y0 + ly * WAVE + s;
              if (y < y0 + TILE - 1 && C(DOWN, x, y) > 0 && Hh(x, y + 1) + 1 < Hh(x, y)) { Hh(x, y) = Hh(x, y + 1) + 1; changed = true; }
            }
          }
        for (int lx = 0; lx < TILE; ++lx)
          for (int ly = 0; ly < NWAVE; ++ly) {
            int y = y0 + lx;
            for (int s = 0; s < WAVE; ++s) {          // left pass
              int x = x0 + ly * WAVE + s;
              if (x > x0 && C(LEFT, x, y) > 0 && Hh(x - 1, y) + 1 < Hh(x, y)) { Hh(x, y) = Hh(x - 1, y) + 1; changed = true; }
            }
            for (int s = WAVE - 1; s >= 0; --s) {     // right pass
              int x = x0 + ly * WAVE + s;
              if (x < x0 + TILE - 1 && C(RIGHT, x, y) > 0 && Hh(x + 1, y) + 1 < Hh(x, y)) { Hh(x, y) = Hh(x + 1, y) + 1; changed = true; }
            }
          }
        ++rounds;
      }
      if (rounds > 1) {
#pragma omp atomic write
        edges.tiles[t] = it_edges;
        if (ty + 1 < TH) {
#pragma omp atomic write
          edges.tiles[t + TW] = it_edges;
        }
        if (tx + 1 < TW) {
#pragma omp atomic write
          edges.tiles[t + 1] = it_edges;
        }
      }
      if (changed) {
#pragma omp atomic write
        bfs.tiles[t] = it_bfs_next;
#pragma omp atomic write
        capped = true;
      }
    }
    return capped;
  }

  // bfs_intertile (graphcut.cl:804-868): relax the top and left edges of each listed tile
  // in both directions and stamp the tiles whose distances changed.
  void intertile(int32_t it) {
    for (int t : edges.list) {
      int tx = t % TW, ty = t / TW;
      bool f0 = false, f1 = false, f2 = false;
      for (int lx = 0; lx < TILE; ++lx) {
        if (ty > 0) {
          int x = tx * TILE + lx, y = ty * TILE;
          bool can = C(UP, x, y) > 0, can2 = C(DOWN, x, y - 1) > 0;
          int32_t d = Hh(x, y), d2 = Hh(x, y - 1);
          if (can && d2 + 1 < d) { Hh(x, y) = d2 + 1; f0 = true; }
          if (can2 && d + 1 < d2) { Hh(x, y - 1) = d + 1; f1 = true; }
        }
        if (tx > 0) {
          int x = tx * TILE, y = ty * TILE + lx;
          bool can = C(LEFT, x, y) > 0, can2 = C(RIGHT, x - 1, y) > 0;
          int32_t d = Hh(x, y), d2 = Hh(x - 1, y);
          if (can && d2 + 1 < d) { Hh(x, y) = d2 + 1; f0 = true; }
          if (can2 && d + 1 < d2) { Hh(x - 1, y) = d + 1; f2 = true; }
        }
      }
      if (f0) bfs.tiles[t] = it;
      if (f1) bfs.tiles[t - TW] = it;
      if (f2) bfs.tiles[t - 1] = it;
    }
  }

  // GraphCut.startBfs (GraphCut.pyx:187-222).  Tiles that hit the in-tile round cap are
  // stamped with the next BFS iteration, so the loop also continues when no edge changed.
  void start_bfs() {
    init_bfs(bfs.increment());
    while (true) {
      bfs.build();
      if (bfs.length() == 0) break;
      ++bfs_rounds;
      bool capped = intratile(edges.increment(), bfs.iteration + 1);
      edges.build();
      if (edges.length() == 0) {
        if (!capped) break;
        bfs.increment();
        continue;
      }
      intertile(bfs.increment());
    }
  }

  // check_completion (graphcut.cl:20-60) + GraphCut.isCompleted (GraphCut.pyx:328-346).
  bool completed() {
    int active = 0;
    const auto& L = load.list;
#pragma omp parallel for reduction(+:active) schedule(static)
    for (int k = 0; k < (int)L.size(); ++k) {
      int t = L[k], tx = t % TW, ty = t / TW;
      for (int y = ty * TILE; y < (ty + 1) * TILE; ++y)
        for (int x = tx * TILE; x < (tx + 1) * TILE; ++x)
          if (E(x, y) > 0 && Hh(x, y) < MAXH) active++;
    }
    return active == 0;
  }

  // GraphCut.cut (GraphCut.pyx:348-418).
  int cut(int bfs_period, long long max_iters) {
    int32_t loadIteration = load.iteration;
    init_gc(load.increment());
    load.build();
    load_tiles(load.list);
    start_bfs();
    long long iteration = 1;
    while (true) {
      if (iteration > max_iters) return 3;  // not converged
      push();
      ++iterations;
      if (iteration % bfs_period == 0) {
        load.increment();
        load.incorporate(brd.tiles, OP_LTE, loadIteration, OP_GTE, brd.iteration - bfs_period * 4, true);
        load.build();
        if (load.length() > 0) load_tiles(load.list);
        load.build(OP_GT, loadIteration);
        start_bfs();
        if (completed()) return 0;
      } else {
        relabel();
        ++relabels;
      }
      ++iteration;
    }
  }
};

}  // namespace

extern "C" {

// Exact max-flow by Boykov-Kolmogorov.  Writes the flow value, the canonical labels
// (1 = source side) and, when final_excess is not null, the final terminal residual.
int orc_maxflow_bk(int W, int H, const int32_t* up, const int32_t* down, const int32_t* left,
                   const int32_t* right, const int32_t* excess, int64_t* flow_out,
                   uint8_t* labels_out, int64_t* final_excess) {
  if (W <= 0 || H <= 0) return 1;
  const int32_t* caps[4] = {up, down, left, right};
  BK bk;
  bk.init(W, H, caps, excess);
  bk.run();
  const int32_t* rc[4] = {bk.rc[0].data(), bk.rc[1].data(), bk.rc[2].data(), bk.rc[3].data()};
  if (labels_out) canonical_labels(bk.g, rc, bk.tr.data(), labels_out);
  int64_t f = flow_value(bk.g.N, excess, bk.tr.data());
  if (f != bk.flow) return 2;  // the two flow accountings must agree
  if (flow_out) *flow_out = f;
  if (final_excess) std::memcpy(final_excess, bk.tr.data(), sizeof(int64_t) * bk.g.N);
  return 0;
}

// Canonical cut of a residual state: labels = reachable from excess > 0 over residual
// edges; flow = sum(max(t0,0)) - sum(max(e,0)).
int orc_canonical(int W, int H, const int32_t* rup, const int32_t* rdown, const int32_t* rleft,
                  const int32_t* rright, const int32_t* exc, const int32_t* t0,
                  int64_t* flow_out, uint8_t* labels_out) {
  Grid g{W, H, (long long)W * H};
  const int32_t* rc[4] = {rup, rdown, rleft, rright};
  std::vector<int64_t> e(exc, exc + g.N);
  if (labels_out) canonical_labels(g, rc, e.data(), labels_out);
  if (flow_out) *flow_out = flow_value(g.N, t0, e.data());
  return 0;
}

// Capacity of the cut whose source side is labels == 1, from the original capacities.
int64_t orc_cut_capacity(int W, int H, const int32_t* up, const int32_t* down,
                         const int32_t* left, const int32_t* right, const int32_t* excess,
                         const uint8_t* labels) {
  Grid g{W, H, (long long)W * H};
  const int32_t* caps[4] = {up, down, left, right};
  int64_t c = 0;
  for (long long i = 0; i < g.N; ++i) {
    if (labels[i]) {
      c += std::max<int64_t>(-(int64_t)excess[i], 0);
      for (int d = 0; d < 4; ++d)
        if (g.has(i, d) && !labels[g.nb(i, d)]) c += caps[d][i];
    } else {
      c += std::max<int64_t>(excess[i], 0);
    }
  }
  return c;
}

// The reference schedule restated (see TiledRef).  W and H must be multiples of 32.
// stats (may be null): [iterations, relabel passes, bfs rounds].
int orc_ref_tiled(int W, int H, const int32_t* up, const int32_t* down, const int32_t* left,
                  const int32_t* right, const int32_t* excess, int bfs_period,
                  long long max_iters, int nthreads, int64_t* flow_out, uint8_t* labels_out,
                  int64_t* stats) {
  if (W <= 0 || H <= 0 || W % 32 || H % 32 || bfs_period <= 0) return 1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const int32_t* caps[4] = {up, down, left, right};
  TiledRef r;
  r.setup(W, H, caps, excess);
  int st = r.cut(bfs_period, max_iters);
  if (stats) { stats[0] = r.iterations; stats[1] = r.relabels; stats[2] = r.bfs_rounds; }
  if (st) return st;
  // tiles that were never loaded keep capacity 0 in the residual planes; their true
  // residual is the uploaded capacity plus the reverse flow already recorded
  for (int t = 0; t < r.NT; ++t) {
    if (r.loaded[t]) continue;
    int tx = t % r.TW, ty = t / r.TW;
    for (int y = ty * 32; y < (ty + 1) * 32; ++y)
      for (int x = tx * 32; x < (tx + 1) * 32; ++x) {
        long long i = (long long)y * W + x;
        for (int d = 0; d < 4; ++d) r.cap[d][i] += r.src[d][i];
      }
  }
  Grid g{W, H, (long long)W * H};
  const int32_t* rc[4] = {r.cap[0].data(), r.cap[1].data(), r.cap[2].data(), r.cap[3].data()};
  std::vector<int64_t> e(r.exc.begin(), r.exc.end());
  if (labels_out) canonical_labels(g, rc, e.data(), labels_out);
  if (flow_out) *flow_out = flow_value(g.N, excess, e.data());
  return 0;
}

}  // extern "C"
