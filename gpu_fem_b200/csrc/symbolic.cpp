// Host-side symbolic setup: block pattern, RCM, elemIndMap, ILU(k) pattern,
// level sets and the coloured scatter schedule.
#include <algorithm>
#include <cstdlib>
#include <random>
#include <cstring>
#include <numeric>

#include "gf_internal.h"

namespace gf {

Pattern pattern_from_conn(int nelem, int nnodes, const int32_t* conn) {
  // Counting pass over element node pairs, then per-row sort/unique.
  Pattern p;
  p.n = nnodes;
  std::vector<int32_t> cnt(nnodes + 1, 0);
  for (int e = 0; e < nelem; e++)
    for (int a = 0; a < 4; a++) cnt[conn[4 * e + a] + 1] += 4;
  for (int i = 0; i < nnodes; i++) cnt[i + 1] += cnt[i];
  std::vector<int32_t> tmp(cnt[nnodes]), fill(cnt.begin(), cnt.end() - 1);
  for (int e = 0; e < nelem; e++)
    for (int a = 0; a < 4; a++) {
      int r = conn[4 * e + a];
      for (int b = 0; b < 4; b++) tmp[fill[r]++] = conn[4 * e + b];
    }
  p.rowp.assign(nnodes + 1, 0);
  p.cols.reserve(cnt[nnodes] / 2 + 1);
  for (int i = 0; i < nnodes; i++) {
    auto b = tmp.begin() + cnt[i], e = tmp.begin() + cnt[i + 1];
    std::sort(b, e);
    auto last = std::unique(b, e);
    p.cols.insert(p.cols.end(), b, last);
    p.rowp[i + 1] = (int32_t)p.cols.size();
  }
  return p;
}

void rcm_order(const Pattern& p, int root, int iters, std::vector<int32_t>& rcm) {
  const int n = p.n;
  rcm.assign(n, -1);
  if (n == 0) return;
  if (iters < 1) iters = 1;
  std::vector<int32_t> levset(n);
  for (int it = 0; it < iters; it++) {
    int start = 0, end = 0, var = 0;
    std::fill(rcm.begin(), rcm.end(), -1);
    while (var < n) {
      if (end - start == 0) {
        if (rcm[root] >= 0) {
          int i = 0;
          for (; i < n; i++)
            if (rcm[i] < 0) break;
          if (i >= n) break;
          root = i;
        }
        levset[end++] = root;
        rcm[root] = var++;
      }
      while (start < end) {
        int next = end;
        for (int cur = start; cur < end; cur++) {
          int node = levset[cur];
          for (int j = p.rowp[node]; j < p.rowp[node + 1]; j++) {
            int nn = p.cols[j];
            if (rcm[nn] < 0) {
              rcm[nn] = var++;
              levset[next++] = nn;
            }
          }
        }
        start = end;
        end = next;
      }
    }
    for (int i = 0; i < var; i++) rcm[levset[i]] = var - 1 - i;
    root = rcm[0];
  }
}

Pattern permute_pattern(const Pattern& p, const std::vector<int32_t>& perm) {
  Pattern q;
  q.n = p.n;
  std::vector<int32_t> iperm(p.n);
  for (int i = 0; i < p.n; i++) iperm[perm[i]] = i;
  q.rowp.assign(p.n + 1, 0);
  q.cols.resize(p.cols.size());
  int nz = 0;
  for (int I = 0; I < p.n; I++) {
    int i = iperm[I], s = nz;
    for (int jp = p.rowp[i]; jp < p.rowp[i + 1]; jp++) q.cols[nz++] = perm[p.cols[jp]];
    std::sort(q.cols.begin() + s, q.cols.begin() + nz);
    q.rowp[I + 1] = nz;
  }
  return q;
}

void elem_ind_map(int nelem, const int32_t* conn, const Pattern& p,
                  const std::vector<int32_t>& perm, std::vector<int32_t>& map) {
  map.assign((size_t)16 * nelem, -1);
  for (int e = 0; e < nelem; e++)
    for (int a = 0; a < 4; a++) {
      int r = perm[conn[4 * e + a]];
      const int32_t* b0 = p.cols.data() + p.rowp[r];
      const int32_t* b1 = p.cols.data() + p.rowp[r + 1];
      for (int b = 0; b < 4; b++) {
        int c = perm[conn[4 * e + b]];
        const int32_t* f = std::lower_bound(b0, b1, c);
        map[16 * e + 4 * a + b] = (f != b1 && *f == c) ? (int32_t)(f - p.cols.data()) : -1;
      }
    }
}

// Bandwidth max |i - j| over the blocks of a pattern (getBandWidth,
// include/linalg/bsr_utils.h:655-670).
int bandwidth(const Pattern& p) {
  int bw = 0;
  for (int i = 0; i < p.n; i++)
    for (int jp = p.rowp[i]; jp < p.rowp[i + 1]; jp++) bw = std::max(bw, std::abs(i - p.cols[jp]));
  return bw;
}

// Deterministic q-ordering (examples/iterative/gmres.cu:159-215, which seeds
// from std::random_device): the RCM order (perm[old] = new) is cut into
// consecutive windows of floor(bandwidth / p) positions, bandwidth that of
// the RCM-ordered pattern, and the positions inside each window are
// permuted at random: a Fisher-Yates shuffle of the window's nodes (new
// position -> node), from its last position down, swapping position i with
// lo + (x mod (i - lo + 1)) for the next 64-bit output x of one MT19937-64
// generator seeded with `seed` for the whole ordering.
void qorder(const Pattern& p, const std::vector<int32_t>& rcm, double pfac, uint64_t seed,
            std::vector<int32_t>& out) {
  const int n = p.n;
  const int bw = bandwidth(permute_pattern(p, rcm));
  const int width = std::max(1, (int)((double)bw / (pfac > 0.0 ? pfac : 1.0)));
  std::vector<int32_t> node(n);  // new position -> node
  for (int i = 0; i < n; i++) node[rcm[i]] = i;
  std::mt19937_64 g(seed);
  for (int lo = 0; lo < n; lo += width) {
    const int hi = std::min(n, lo + width);
    for (int i = hi - 1; i > lo; i--) {
      const int j = lo + (int)(g() % (uint64_t)(i - lo + 1));
      std::swap(node[i], node[j]);
    }
  }
  out.assign(n, 0);
  for (int k = 0; k < n; k++) out[node[k]] = k;
}

Pattern iluk_pattern(const Pattern& a, int lev) {
  Pattern o;
  o.n = a.n;
  o.rowp.assign(a.n + 1, 0);
  std::vector<int32_t> lv, diag(a.n), rcols, rlevs;
  for (int i = 0; i < a.n; i++) {
    rcols.assign(a.cols.begin() + a.rowp[i], a.cols.begin() + a.rowp[i + 1]);
    rlevs.assign(rcols.size(), 0);
    auto it = std::lower_bound(rcols.begin(), rcols.end(), i);
    if (it == rcols.end() || *it != i) {
      rlevs.insert(rlevs.begin() + (it - rcols.begin()), 0);
      rcols.insert(it, i);
    }
    size_t j = 0;
    for (; rcols[j] < i; j++) {
      int k = rcols[j], clev = rlevs[j];
      size_t pp = j + 1;
      for (int kk = diag[k] + 1; kk < o.rowp[k + 1]; kk++) {
        while (pp < rcols.size() && rcols[pp] < o.cols[kk]) pp++;
        int nl = clev + lv[kk] + 1;
        if (pp < rcols.size() && rcols[pp] == o.cols[kk]) {
          if (rlevs[pp] > nl) rlevs[pp] = nl;
        } else if (nl <= lev) {
          rcols.insert(rcols.begin() + pp, o.cols[kk]);
          rlevs.insert(rlevs.begin() + pp, nl);
        }
      }
    }
    diag[i] = o.rowp[i] + (int)j;
    o.cols.insert(o.cols.end(), rcols.begin(), rcols.end());
    lv.insert(lv.end(), rlevs.begin(), rlevs.end());
    o.rowp[i + 1] = (int32_t)o.cols.size();
  }
  return o;
}

int levels(const Pattern& p, bool lower, std::vector<int32_t>& level) {
  level.assign(p.n, 0);
  int nl = 0;
  if (lower) {
    for (int i = 0; i < p.n; i++) {
      int l = 0;
      for (int jp = p.rowp[i]; jp < p.rowp[i + 1] && p.cols[jp] < i; jp++)
        l = std::max(l, level[p.cols[jp]] + 1);
      level[i] = l;
      nl = std::max(nl, l + 1);
    }
  } else {
    for (int i = p.n - 1; i >= 0; i--) {
      int l = 0;
      for (int jp = p.rowp[i]; jp < p.rowp[i + 1]; jp++)
        if (p.cols[jp] > i) l = std::max(l, level[p.cols[jp]] + 1);
      level[i] = l;
      nl = std::max(nl, l + 1);
    }
  }
  return nl;
}

// Scatter schedule.
//  1. Chunks (one warp's work, at most chunk_size elements): seeds in
//     ascending element order; a chunk grows breadth-first over elements
//     sharing a node (neighbours of a node in ascending element order, nodes
//     in element-local order) until it holds chunk_size elements.
//  2. Chunk colours: greedy in chunk order, smallest colour not used by an
//     already-coloured chunk that shares a node. Chunks of one colour share
//     no node and run concurrently.
//  3. Inside a chunk one warp processes the elements one after another in
//     BFS order; an element's "colour" is its position in the chunk.
//  4. Execution order: chunk colour, chunk id, position. The first touch of
//     a matrix block (or residual node) is the toucher with the smallest
//     (chunk colour, position); it stores, later touchers read-modify-write.
int build_schedule(int nelem, int nnodes, const int32_t* conn, const std::vector<int32_t>& emap,
                   int nnzb, int chunk_size, Schedule& s) {
  if (chunk_size > kMaxEC) return -1;
  s.chunk_size = chunk_size;
  // node -> elements
  std::vector<int32_t> ne_ptr(nnodes + 1, 0), ne_idx((size_t)4 * nelem);
  for (int e = 0; e < nelem; e++)
    for (int a = 0; a < 4; a++) ne_ptr[conn[4 * e + a] + 1]++;
  for (int i = 0; i < nnodes; i++) ne_ptr[i + 1] += ne_ptr[i];
  {
    std::vector<int32_t> f(ne_ptr.begin(), ne_ptr.end() - 1);
    for (int e = 0; e < nelem; e++)
      for (int a = 0; a < 4; a++) ne_idx[f[conn[4 * e + a]]++] = e;
  }
  // 1. chunks
  s.elem_chunk.assign(nelem, -1);
  std::vector<int32_t> bfs;  // elements in chunk order, chunk by chunk
  bfs.reserve(nelem);
  std::vector<int32_t> cstart;
  int nc = 0;
  for (int seed = 0; seed < nelem; seed++) {
    if (s.elem_chunk[seed] >= 0) continue;
    size_t head = bfs.size();
    cstart.push_back((int32_t)head);
    s.elem_chunk[seed] = nc;
    bfs.push_back(seed);
    int count = 1;
    while (head < bfs.size() && count < chunk_size) {
      int e = bfs[head++];
      for (int a = 0; a < 4 && count < chunk_size; a++) {
        int n = conn[4 * e + a];
        for (int k = ne_ptr[n]; k < ne_ptr[n + 1] && count < chunk_size; k++) {
          int f = ne_idx[k];
          if (s.elem_chunk[f] < 0) {
            s.elem_chunk[f] = nc;
            bfs.push_back(f);
            count++;
          }
        }
      }
    }
    nc++;
  }
  cstart.push_back((int32_t)bfs.size());
  s.nchunks = nc;
  // 2. chunk colours
  s.chunk_color.assign(nc, -1);
  s.ncc = 0;
  std::vector<char> used;
  for (int c = 0; c < nc; c++) {
    used.assign(used.size(), 0);
    for (int k = cstart[c]; k < cstart[c + 1]; k++) {
      int e = bfs[k];
      for (int a = 0; a < 4; a++) {
        int n = conn[4 * e + a];
        for (int q = ne_ptr[n]; q < ne_ptr[n + 1]; q++) {
          int oc = s.elem_chunk[ne_idx[q]];
          int col = s.chunk_color[oc];
          if (oc != c && col >= 0) {
            if ((int)used.size() <= col) used.resize(col + 1, 0);
            used[col] = 1;
          }
        }
      }
    }
    int col = 0;
    while (col < (int)used.size() && used[col]) col++;
    s.chunk_color[c] = col;
    s.ncc = std::max(s.ncc, col + 1);
  }
  // 3. position inside the chunk
  s.elem_color.assign(nelem, -1);
  s.max_ec = 0;
  for (int c = 0; c < nc; c++)
    for (int k = cstart[c]; k < cstart[c + 1]; k++) {
      s.elem_color[bfs[k]] = k - cstart[c];
      s.max_ec = std::max(s.max_ec, k - cstart[c] + 1);
    }
  // 4. execution order
  s.chunk_list.resize(nc);
  std::iota(s.chunk_list.begin(), s.chunk_list.end(), 0);
  std::stable_sort(s.chunk_list.begin(), s.chunk_list.end(),
                   [&](int x, int y) { return s.chunk_color[x] < s.chunk_color[y]; });
  s.cc_start.assign(s.ncc + 1, 0);
  for (int c = 0; c < nc; c++) s.cc_start[s.chunk_color[c] + 1]++;
  for (int k = 0; k < s.ncc; k++) s.cc_start[k + 1] += s.cc_start[k];
  s.order.clear();
  s.order.reserve(nelem);
  s.chunk_start.assign(nc + 1, 0);
  for (int li = 0; li < nc; li++) {
    int c = s.chunk_list[li];
    s.chunk_start[li] = (int32_t)s.order.size();
    for (int k = cstart[c]; k < cstart[c + 1]; k++) s.order.push_back(bfs[k]);
  }
  s.chunk_start[nc] = (int32_t)s.order.size();
  // first-touch masks
  const int stride = kMaxEC + 1;
  std::vector<int32_t> tb(nnzb, INT32_MAX), tn(nnodes, INT32_MAX);
  for (int e = 0; e < nelem; e++) {
    int t = s.chunk_color[s.elem_chunk[e]] * stride + s.elem_color[e];
    for (int k = 0; k < 16; k++) tb[emap[16 * e + k]] = std::min(tb[emap[16 * e + k]], t);
    for (int a = 0; a < 4; a++) tn[conn[4 * e + a]] = std::min(tn[conn[4 * e + a]], t);
  }
  s.first_touch.assign(nelem, 0);
  for (int e = 0; e < nelem; e++) {
    int t = s.chunk_color[s.elem_chunk[e]] * stride + s.elem_color[e];
    uint32_t m = 0;
    for (int k = 0; k < 16; k++)
      if (tb[emap[16 * e + k]] == t) m |= 1u << k;
    for (int a = 0; a < 4; a++)
      if (tn[conn[4 * e + a]] == t) m |= 1u << (16 + a);
    s.first_touch[e] = m;
  }
  return 0;
}

}  // namespace gf

namespace gf {
void order_nodes(const Pattern& p, const gf_mesh_desc* d, std::vector<int32_t>& perm) {
  if (d->ordering == GF_ORDER_RCM || d->ordering == GF_ORDER_QORDER) {
    rcm_order(p, d->rcm_root, 1, perm);
    if (d->ordering == GF_ORDER_QORDER) {
      std::vector<int32_t> q;
      qorder(p, perm, d->qorder_p, d->qorder_seed, q);
      perm.swap(q);
    }
  } else {
    perm.resize(p.n);
    for (int i = 0; i < p.n; i++) perm[i] = i;
  }
}
}  // namespace gf

extern "C" gf_status gf_order_nodes(const gf_mesh_desc* d, int32_t* perm) {
  if (!d || !perm || d->num_nodes <= 0 || d->num_elements < 0 || !d->conn ||
      d->ordering < GF_ORDER_NATURAL || d->ordering > GF_ORDER_QORDER)
    return GF_INVALID_ARG;
  for (int i = 0; i < 4 * d->num_elements; i++)
    if (d->conn[i] < 0 || d->conn[i] >= d->num_nodes) return GF_INVALID_ARG;
  if (d->rcm_root < 0 || d->rcm_root >= d->num_nodes) return GF_INVALID_ARG;
  const gf::Pattern p = gf::pattern_from_conn(d->num_elements, d->num_nodes, d->conn);
  std::vector<int32_t> v;
  gf::order_nodes(p, d, v);
  std::copy(v.begin(), v.end(), perm);
  return GF_OK;
}
