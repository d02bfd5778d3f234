// Host symbolic analysis (see symbolic.h).
//
// The ordering and the supernode partition decide which pivots the numeric
// phase sees, so they have to reproduce the reference's arrays exactly.  The
// steps below therefore follow the reference's algorithms step for step
// (same quotient-graph storage, same bucket order for equal degrees, same
// tie-breaking sort in the supernode relaxation), written independently.
// Reference: include/block_amd.h, include/ordering_utils.h:313-360, 812-838,
// include/sparse_ldl.h:2204-3104.
#include "symbolic.h"

#include <algorithm>
#include <cstdio>
#include <numeric>

namespace ab {
namespace {

// ---------------------------------------------------------------------------
// Sorted, de-duplicated integer list helper used by the degree machinery:
// sorts a[0:len], drops negative entries and repeated values, returns the new
// length.  (block_amd.h:457-476)
int sort_unique_nonneg(int len, int* a) {
  std::sort(a, a + len);
  int src = 0, dst = 0;
  while (src < len && a[src] < 0) src++;
  for (; src < len; src++, dst++) {
    while (src < len - 1 && a[src] == a[src + 1]) src++;
    if (src != dst) a[dst] = a[src];
  }
  return dst;
}

// Degree buckets with LIFO insertion (block_amd.h:687-812).  The minimum
// degree pointer only moves down; lookups scan upward from it.
struct DegreeBuckets {
  int size;
  int floor_deg;
  std::vector<int> deg, head, nxt, prv;

  DegreeBuckets(int n, const int* rowp)
      : size(n), deg(n), head(n + 1, -1), nxt(n + 1, -1), prv(n + 1, -1) {
    floor_deg = 0;
    for (int v = 0; v < n; v++) {
      deg[v] = rowp[v + 1] - rowp[v];
      if (v == 0 || deg[v] < floor_deg) floor_deg = deg[v];
    }
    for (int v = 0; v < n; v++) push_front(v, deg[v]);
  }
  void push_front(int v, int d) {
    if (head[d] != -1) {
      prv[head[d]] = v;
      nxt[v] = head[d];
    }
    head[d] = v;
  }
  void unlink(int v) {
    int d = deg[v];
    if (head[d] == v) head[d] = nxt[v];
    if (nxt[v] != -1) prv[nxt[v]] = prv[v];
    if (prv[v] != -1) nxt[prv[v]] = nxt[v];
    prv[v] = nxt[v] = -1;
  }
  void set(int v, int d) {
    if (d < floor_deg) floor_deg = d;
    unlink(v);
    push_front(v, d);
    deg[v] = d;
  }
  int pick() const {
    for (int d = floor_deg; d <= size; d++)
      if (head[d] != -1) return head[d];
    return -1;
  }
};

// Quotient graph: row r of `adj` holds [elements (elen) | variables] in the
// slot rowp[r] .. rowp[r+1]; alen is the used length.  Elements and
// variables are kept sorted inside their sections.
struct QuotientGraph {
  int n;
  std::vector<int>& rowp;
  std::vector<int>& adj;
  std::vector<int> alen, elen;

  QuotientGraph(int n_, std::vector<int>& rp, std::vector<int>& a)
      : n(n_), rowp(rp), adj(a), alen(n_), elen(n_, 0) {
    for (int v = 0; v < n; v++) alen[v] = rowp[v + 1] - rowp[v];
  }
  int* row(int r) { return adj.data() + rowp[r]; }
  int cap(int r) const { return rowp[r + 1] - rowp[r]; }

  // Make `need` more slots available at the end of row r by compacting
  // neighbouring rows: first the rows below r (toward 0), then the rows
  // above it.  (block_amd.h:519-580)
  void grow_row(int r, int need) {
    int got = 0;
    if (r > 0) {
      int s = r - 1;
      for (; got < need && s >= 0; s--) got += cap(s) - alen[s];
      s++;
      int dst = rowp[s] + alen[s];
      for (int q = s + 1; q <= r; q++) {
        int src = rowp[q];
        int start = dst;
        for (int e = src + alen[q]; src < e; src++, dst++) adj[dst] = adj[src];
        rowp[q] = start;
      }
    }
    if (got < need) {
      int s = r + 1;
      for (; got < need && s < n; s++) got += cap(s) - alen[s];
      s--;
      if (s >= n) {
        s = n - 1;
        std::fprintf(stderr, "amd: quotient graph storage exhausted\n");
      }
      int dst = rowp[s + 1] - 1;
      for (int q = s; q > r; q--) {
        int lo = rowp[q];
        for (int src = lo + alen[q] - 1; src >= lo; src--, dst--)
          adj[dst] = adj[src];
        rowp[q] = rowp[q + 1] - alen[q];
      }
    }
  }

  // True when variables a and b have identical adjacency once each is
  // allowed to skip the other (block_amd.h:597-626).
  bool same_adjacency(int a, int b) const {
    if (a == b) return false;
    if (alen[a] != alen[b] || elen[a] != elen[b]) return false;
    int len = alen[a];
    int pa = rowp[a], ea = pa + alen[a];
    int pb = rowp[b], eb = pb + alen[b];
    for (int t = 0; t < len; t++, pa++, pb++) {
      if (adj[pa] == b) pa++;
      if (adj[pb] == a) pb++;
      if (adj[pa] != adj[pb]) break;
    }
    return pa == ea && pb == eb;
  }

  // Drop variable v from every element and variable list that names it
  // (block_amd.h:633-674).
  void detach(int v) {
    int p = rowp[v];
    for (; p < rowp[v] + elen[v]; p++) {
      int e = adj[p];
      int q = rowp[e], last = rowp[e] + alen[e] - 1;
      while (q < last && adj[q] != v) q++;
      for (; q < last; q++) adj[q] = adj[q + 1];
      alen[e]--;
    }
    for (; p < rowp[v] + alen[v]; p++) {
      int w = adj[p];
      int q = rowp[w] + elen[w], last = rowp[w] + alen[w] - 1;
      while (q < last && adj[q] != v) q++;
      for (; q < last; q++) adj[q] = adj[q + 1];
      alen[w]--;
    }
    elen[v] = alen[v] = 0;
  }
};

}  // namespace

// Approximate minimum degree, following include/block_amd.h:27-452 with no
// multiplier block (the reference calls it with nmult = 0 from
// OrderingUtils::amd, include/ordering_utils.h:202-221).
int amd_order(int n, std::vector<int>& rowp, std::vector<int>& adj,
              std::vector<int>& perm) {
  perm.resize(n);
  QuotientGraph G(n, rowp, adj);
  std::vector<int> svsize(n, 1);     // supervariable size, -(rep+1) if merged
  std::vector<int> status(n, 1);     // 1 variable, 0 pivot, -1 absorbed
  std::vector<int> edeg(n, -1);      // cached |element \ current var|
  std::vector<int> Lp(n);
  for (int v = 0; v < n; v++) perm[v] = v;

  // Input rows must be strictly increasing and non-negative.
  for (int v = 0; v < n; v++) {
    const int* r = G.row(v);
    for (int t = 0; t + 1 < G.alen[v]; t++)
      if (r[t] < 0 || r[t + 1] < 0 || r[t + 1] <= r[t]) return 1;
  }

  DegreeBuckets B(n, rowp.data());
  int npiv = 0;
  for (int elim = 0; elim < n; npiv++) {
    const int piv = B.pick();
    B.unlink(piv);
    perm[npiv] = piv;
    status[piv] = 0;

    // Lp = {piv} U vars(piv) U vars of every element adjacent to piv.
    int nl = 0;
    Lp[nl++] = piv;
    for (int p = rowp[piv] + G.elen[piv]; p < rowp[piv] + G.alen[piv]; p++)
      if (adj[p] != piv) Lp[nl++] = adj[p];
    for (int p = rowp[piv]; p < rowp[piv] + G.elen[piv]; p++) {
      int e = adj[p];
      for (int q = rowp[e] + G.elen[e]; q < rowp[e] + G.alen[e]; q++) {
        if (nl >= n) nl = sort_unique_nonneg(nl, Lp.data());
        if (adj[q] != piv) Lp[nl++] = adj[q];
      }
    }
    nl = sort_unique_nonneg(nl, Lp.data());

    // Element absorption and removal of Lp from each neighbour's var list.
    for (int t = 0; t < nl; t++) {
      const int w = Lp[t];
      if (w == piv) continue;
      int absorbed = 0, dropped = 0;
      const int pe_end = rowp[piv] + G.elen[piv];
      for (int k = rowp[piv], c = rowp[w];
           k < pe_end && c < rowp[w] + G.elen[w]; c++) {
        while (k < pe_end && adj[k] < adj[c]) k++;
        if (k < pe_end && adj[k] == adj[c]) {
          adj[c] = -1;
          absorbed++;
        }
      }
      for (int k = 0, c = rowp[w] + G.elen[w];
           k < nl && c < rowp[w] + G.alen[w]; c++) {
        while (k < nl && Lp[k] < adj[c]) k++;
        if (k < nl && adj[c] == Lp[k]) {
          adj[c] = -1;
          dropped++;
        }
      }
      if (absorbed > 0 || dropped > 0) {
        int end = rowp[w] + G.alen[w];
        int src = rowp[w], dst = src;
        for (; src < end; src++, dst++) {
          while (src < end && adj[src] == -1) src++;
          if (src < end) adj[dst] = adj[src];
        }
        G.elen[w] -= absorbed;
        G.alen[w] -= absorbed + dropped;
      }
    }

    // piv becomes an element of every neighbour (sorted insertion).
    for (int t = 0; t < nl; t++) {
      const int w = Lp[t];
      if (w == piv) continue;
      if (G.alen[w] == G.cap(w)) G.grow_row(w, 1);
      int k = rowp[w];
      const int e_end = k + G.elen[w];
      while (k < e_end && adj[k] < piv) k++;
      if (adj[k] != piv) {
        for (int p = rowp[w] + G.alen[w] - 1; p >= k; p--) adj[p + 1] = adj[p];
        adj[k] = piv;
        G.alen[w]++;
        G.elen[w]++;
      }
    }

    // Elements adjacent to piv are absorbed into the new element piv.
    for (int p = rowp[piv]; p < rowp[piv] + G.elen[piv]; p++) {
      int e = adj[p];
      G.alen[e] = 0;
      G.elen[e] = 0;
      status[e] = -1;
    }

    // Row piv now stores the variable list Lp \ {piv}.
    if (nl - 1 > G.cap(piv)) G.grow_row(piv, nl - 1 - G.cap(piv));
    G.elen[piv] = 0;
    G.alen[piv] = nl - 1;
    for (int p = rowp[piv], k = 0; k < nl; k++, p++) {
      if (Lp[k] == piv) {
        k++;
        if (k == nl) break;
      }
      adj[p] = Lp[k];
    }

    // Approximate external degrees (block_amd.h:267-374).
    for (int t = 0; t < nl; t++) {
      const int w = Lp[t];
      for (int p = rowp[w]; p < rowp[w] + G.elen[w]; p++) {
        int e = adj[p];
        if (edeg[e] < 0) {
          edeg[e] = 0;
          for (int q = rowp[e]; q < rowp[e] + G.alen[e]; q++)
            edeg[e] += svsize[adj[q]];
        }
        edeg[e] -= svsize[w];
      }
    }
    int lp_weight = 0;
    for (int t = 0; t < nl; t++)
      if (Lp[t] != piv) lp_weight += svsize[Lp[t]];
    for (int t = 0; t < nl; t++) {
      const int w = Lp[t];
      if (w == piv) continue;
      int est = lp_weight;
      for (int p = rowp[w] + G.elen[w]; p < rowp[w] + G.alen[w]; p++)
        est += svsize[adj[p]];
      const int vstart = rowp[w] + G.elen[w];
      const int vlen = G.alen[w] - G.elen[w];
      if (vlen > 0 &&
          std::binary_search(adj.data() + vstart, adj.data() + vstart + vlen, w))
        est -= svsize[w];
      if (std::binary_search(Lp.data(), Lp.data() + nl, w)) est -= svsize[w];
      for (int p = rowp[w]; p < rowp[w] + G.elen[w]; p++) {
        int e = adj[p];
        if (e == piv) continue;
        if (edeg[e] < 0) {
          edeg[e] = 0;
          for (int q = rowp[e]; q < rowp[e] + G.alen[e]; q++)
            edeg[e] += svsize[adj[q]];
        }
        est += edeg[e];
      }
      est = est < n - elim ? est : n - elim;
      int d = B.deg[w];
      d = est < d + lp_weight ? est : d + lp_weight;
      B.set(w, d);
    }
    for (int t = 0; t < nl; t++) {
      const int w = Lp[t];
      for (int p = rowp[w]; p < rowp[w] + G.elen[w]; p++) edeg[adj[p]] = -1;
    }

    // Indistinguishable neighbours collapse into supervariables.
    for (int a = 0; a < nl; a++) {
      const int u = Lp[a];
      if (u == piv || svsize[u] < 0) continue;
      for (int b = a + 1; b < nl; b++) {
        const int v = Lp[b];
        if (v == piv || svsize[v] < 0) continue;
        if (G.same_adjacency(u, v)) {
          svsize[u] += svsize[v];
          B.set(u, B.deg[u] - svsize[v]);
          svsize[v] = -(u + 1);
          status[v] = -1;
          G.detach(v);
          B.unlink(v);
        }
      }
    }
    elim += svsize[piv];
  }

  // Expand supervariables: representatives in pivot order, members right
  // after their representative in increasing index order.
  int end = n;
  for (int j = npiv - 1; j >= 0; j--) {
    int sv = perm[j];
    end -= svsize[sv];
    perm[end] = sv;
    status[sv] = end + 1;
  }
  for (int v = 0; v < n; v++) {
    if (svsize[v] < 0) {
      int r = v;
      while (svsize[r] < 0) r = -(svsize[r] + 1);
      perm[status[r]] = v;
      status[r]++;
    }
  }
  return 0;
}

// Pattern copy for the ordering step (ordering_utils.h:313-360) followed by
// the in-place sort/uniquify (ordering_utils.h:812-838).
static void ordering_pattern(int order, int n, const int* rowp,
                             const int* cols, std::vector<int>& rp,
                             std::vector<int>& cc) {
  rp.assign(n + 1, 0);
  if (order == ORDER_ND) {
    cc.assign(rowp[n], 0);
    int ptr = 0;
    for (int i = 0; i < n; i++) {
      for (int p = rowp[i]; p < rowp[i + 1]; p++)
        if (cols[p] != i) cc[ptr++] = cols[p];
      rp[i + 1] = ptr;
    }
  } else {
    cc.assign(rowp[n] + n, 0);
    int ptr = 0;
    for (int i = 0; i < n; i++) {
      cc[ptr++] = i;
      for (int p = rowp[i]; p < rowp[i + 1]; p++) cc[ptr++] = cols[p];
      rp[i + 1] = ptr;
    }
  }
  int start = rp[0];
  for (int i = 0; i < n; i++) {
    int len = rp[i + 1] - start;
    int* seg = cc.data() + start;
    std::sort(seg, seg + len);
    int keep = 0;
    if (len > 0) {
      cc[rp[i]] = seg[0];
      keep = 1;
      for (int t = 1; t < len; t++)
        if (seg[t] != cc[rp[i] + keep - 1]) cc[rp[i] + keep++] = seg[t];
    }
    start = rp[i + 1];
    rp[i + 1] = rp[i] + keep;
  }
}

void compute_ordering(int order, int n, const int* rowp, const int* cols,
                      std::vector<int>& perm, std::vector<int>& iperm) {
  perm.assign(n, 0);
  iperm.assign(n, 0);
  if (order == ORDER_AMD) {
    std::vector<int> rp, cc;
    ordering_pattern(order, n, rowp, cols, rp, cc);
    if (amd_order(n, rp, cc, perm) != 0)
      std::fprintf(stderr, "amd: malformed input pattern\n");
    for (int i = 0; i < n; i++) iperm[perm[i]] = i;
  } else if (order == ORDER_MULTI_COLOR) {
    // The reference's multi-colour path reads an uninitialised permutation
    // (include/ordering_utils.h:281-291); it has no defined result to
    // reproduce, so it is rejected by the caller.
    for (int i = 0; i < n; i++) perm[i] = iperm[i] = i;
  } else {
    // NESTED_DISSECTION without METIS is the identity
    // (include/ordering_utils.h:177-197), as is NATURAL.
    for (int i = 0; i < n; i++) perm[i] = iperm[i] = i;
  }
}

namespace {

// Elimination tree with path-compressed ancestors (sparse_ldl.h:2375-2440).
void etree(int n, const int* rowp, const int* cols, const int* perm,
           const int* iperm, std::vector<int>& parent) {
  std::vector<int> anc(n, -1);
  parent.assign(n, -1);
  for (int k = 0; k < n; k++) {
    const int ka = perm ? perm[k] : k;
    for (int p = rowp[ka]; p < rowp[ka + 1]; p++) {
      int i = perm ? iperm[cols[p]] : cols[p];
      while (i < k) {
        int up = anc[i];
        anc[i] = k;
        if (up == -1) {
          parent[i] = k;
          break;
        }
        i = up;
      }
    }
  }
}

// Depth-first post-order of the forest; children are visited in increasing
// index order (sparse_ldl.h:2455-2518).
void postorder(int n, const std::vector<int>& parent, std::vector<int>& post) {
  std::vector<int> head(n, -1), next(n, -1), stack(n);
  post.assign(n, 0);
  for (int j = n - 1; j >= 0; j--) {
    if (parent[j] != -1) {
      next[j] = head[parent[j]];
      head[parent[j]] = j;
    }
  }
  int k = 0;
  for (int root = 0; root < n; root++) {
    if (parent[root] != -1) continue;
    int top = 0;
    stack[0] = root;
    while (top >= 0) {
      int p = stack[top];
      int c = head[p];
      if (c == -1) {
        post[k++] = p;
        top--;
      } else {
        head[p] = next[c];
        stack[++top] = c;
      }
    }
  }
}

// Column counts of L by the row-subtree / least-common-ancestor method
// (sparse_ldl.h:2560-2701).
void column_counts(int n, const int* rowp, const int* cols, const int* perm,
                   const int* iperm, const std::vector<int>& parent,
                   const std::vector<int>& post, std::vector<int>& cnt) {
  std::vector<int> first(n, -1), prevleaf(n, -1), maxfirst(n, -1), anc(n);
  cnt.assign(n, 0);
  for (int k = 0; k < n; k++) {
    int j = post[k];
    if (first[j] == -1) cnt[j] = 1;
    while (j != -1 && first[j] == -1) {
      first[j] = k;
      j = parent[j];
    }
  }
  std::iota(anc.begin(), anc.end(), 0);
  auto find = [&](int p) {
    int r = p;
    while (anc[r] != r) r = anc[r];
    while (anc[p] != p) {
      int nx = anc[p];
      anc[p] = r;
      p = nx;
    }
    return r;
  };
  for (int k = 0; k < n; k++) {
    const int j = post[k];
    const int ja = perm ? perm[j] : j;
    if (parent[j] != -1) cnt[parent[j]]--;
    for (int p = rowp[ja]; p < rowp[ja + 1]; p++) {
      const int i = perm ? iperm[cols[p]] : cols[p];
      if (i <= j) continue;
      if (first[j] <= maxfirst[i]) continue;
      cnt[j]++;
      maxfirst[i] = first[j];
      const int jprev = prevleaf[i];
      prevleaf[i] = j;
      if (jprev != -1) cnt[find(jprev)]--;
    }
    if (parent[j] != -1) anc[j] = parent[j];
  }
  for (int k = 0; k < n; k++) {
    const int j = post[k];
    if (parent[j] != -1) cnt[parent[j]] += cnt[j];
  }
}

// Children lists with all roots appended after the last node
// (sparse_ldl.h:2960-2996).
void children_lists(int nn, const int* par, std::vector<int>& cptr,
                    std::vector<int>& kids) {
  cptr.assign(nn + 2, 0);
  kids.assign(nn, 0);
  for (int i = 0; i < nn; i++) cptr[(par[i] != -1 ? par[i] : nn) + 1]++;
  for (int i = 0; i < nn + 1; i++) cptr[i + 1] += cptr[i];
  for (int i = 0; i < nn; i++) {
    int slot = par[i] != -1 ? par[i] : nn;
    kids[cptr[slot]++] = i;
  }
  for (int i = nn; i >= 0; i--) cptr[i + 1] = cptr[i];
  cptr[0] = 0;
}

}  // namespace

void analyze(int order, int n, const int* rowp, const int* cols,
             SymbolicTree& T) {
  T = SymbolicTree();
  T.n = n;
  std::vector<int> perm, iperm;
  const int* P = nullptr;
  const int* IP = nullptr;
  if (order != ORDER_NATURAL) {
    compute_ordering(order, n, rowp, cols, perm, iperm);
    P = perm.data();
    IP = iperm.data();
    T.permuted = true;
  }

  std::vector<int> parent, post, cnt;
  etree(n, rowp, cols, P, IP, parent);
  postorder(n, parent, post);
  column_counts(n, rowp, cols, P, IP, parent, post, cnt);

  // Fundamental supernodes: chains along the post-order whose column counts
  // drop by exactly one (sparse_ldl.h:2716-2747).
  std::vector<int> v2s(n), s2v(n);
  int ns = 0;
  for (int i = 0; i < n; ns++) {
    int v = post[i];
    v2s[v] = ns;
    s2v[i] = v;
    i++;
    int nxt = i < n ? post[i] : n;
    while (i < n && parent[v] == nxt && cnt[nxt] == cnt[v] - 1) {
      v = nxt;
      v2s[v] = ns;
      s2v[i] = v;
      i++;
      if (i < n) nxt = post[i];
    }
  }
  std::vector<int> sptr(ns + 1, 0);
  for (int i = 0; i < n; i++) sptr[v2s[i] + 1]++;
  for (int s = 0; s < ns; s++) sptr[s + 1] += sptr[s];
  std::vector<int> spar(ns);
  for (int s = 0; s < ns; s++) {
    int p = parent[s2v[sptr[s + 1] - 1]];
    spar[s] = p >= 0 ? v2s[p] : -1;
  }
  std::vector<int> scptr, skids;
  children_lists(ns, spar.data(), scptr, skids);

  // Relaxed supernodes: merge children into parents while the merged width
  // stays <= 64 and the explicit zeros added stay <= 256
  // (sparse_ldl.h:2768-2949).  The children of each supernode are visited in
  // the order std::sort produces for the reference's key, which is the
  // width of the merge group rooted at the child's *position* in the
  // children array; that ordering is reproduced as is.
  const int kMaxWidth = 64, kMaxZeros = 256;
  std::vector<int> rootof(ns), rcnt(ns), width(ns), zeros(ns, 0);
  for (int s = 0; s < ns; s++) {
    width[s] = sptr[s + 1] - sptr[s];
    rcnt[s] = cnt[s2v[sptr[s]]];
    rootof[s] = s;
  }
  auto find = [&](int s) {
    while (rootof[s] != s) {
      rootof[s] = rootof[rootof[s]];
      s = rootof[s];
    }
    return s;
  };
  for (int s = 0; s < ns; s++) {
    std::vector<int> order_pos(scptr[s + 1] - scptr[s]);
    for (int q = scptr[s], t = 0; q < scptr[s + 1]; q++, t++) order_pos[t] = q;
    std::sort(order_pos.begin(), order_pos.end(), [&](int a, int b) {
      return width[find(a)] < width[find(b)];
    });
    for (size_t t = 0; t < order_pos.size(); t++) {
      const int child = skids[order_pos[t]];
      const int rp = find(s), rc = find(child);
      const int merged = width[rc] + width[rp];
      if (rc != rp && merged <= kMaxWidth) {
        int extra = std::max(0, rcnt[rp] - (rcnt[rc] - width[rp]));
        int added = extra * width[rc];
        if (zeros[rp] + zeros[rc] + added <= kMaxZeros) {
          rcnt[rp] = merged + rcnt[rp] - width[rp];
          width[rp] = merged;
          rootof[rc] = rp;
          zeros[rp] += added + zeros[rc];
        }
      }
    }
  }
  std::vector<int> s2n(ns, -1), rep_index(ns, -1);
  int nn = 0;
  for (int s = 0; s < ns; s++)
    if (find(s) == s) rep_index[s] = nn++;
  for (int s = 0; s < ns; s++) s2n[s] = rep_index[find(s)];

  T.num_nodes = nn;
  T.node_ptr.assign(nn + 1, 0);
  T.node_to_var.assign(n, 0);
  std::vector<int> v2n(n), ncnt(nn);
  for (int s = 0; s < ns; s++) T.node_ptr[s2n[s] + 1] += sptr[s + 1] - sptr[s];
  for (int k = 0; k < nn; k++) T.node_ptr[k + 1] += T.node_ptr[k];
  {
    std::vector<int> fill(T.node_ptr.begin(), T.node_ptr.end() - 1);
    for (int s = 0; s < ns; s++) {
      int k = s2n[s];
      for (int q = sptr[s]; q < sptr[s + 1]; q++) {
        int v = s2v[q];
        T.node_to_var[fill[k]++] = v;
        v2n[v] = k;
      }
    }
  }
  for (int s = 0; s < ns; s++) ncnt[s2n[s]] = rcnt[find(s)];
  T.node_parent.assign(nn, -1);
  for (int s = 0; s < ns; s++) {
    int r = find(s);
    if (r != s) continue;
    int k = s2n[r];
    int ps = spar[r];
    if (ps >= 0) {
      int kp = s2n[find(ps)];
      if (kp != k) T.node_parent[k] = kp;
    }
  }
  children_lists(nn, T.node_parent.data(), T.children_ptr, T.children);

  // Contribution rows (rows of L strictly below each node), gathered by the
  // row-subtree walk of every A(i, k), i < k (sparse_ldl.h:3018-3104).
  T.contrib_ptr.assign(nn + 1, 0);
  for (int k = 0; k < nn; k++)
    T.contrib_ptr[k + 1] = ncnt[k] - (T.node_ptr[k + 1] - T.node_ptr[k]);
  for (int k = 0; k < nn; k++) T.contrib_ptr[k + 1] += T.contrib_ptr[k];
  T.contrib_rows.assign(T.contrib_ptr[nn], 0);
  {
    std::vector<int> fillc(nn, 0), flag(nn, -1), npar(nn);
    for (int k = 0; k < nn; k++) {
      int last = T.node_to_var[T.node_ptr[k + 1] - 1];
      int p = parent[last];
      npar[k] = p >= 0 ? v2n[p] : -1;
    }
    for (int k = 0; k < n; k++) {
      const int kn = v2n[k];
      const int ka = P ? P[k] : k;
      for (int p = rowp[ka]; p < rowp[ka + 1]; p++) {
        const int i = P ? IP[cols[p]] : cols[p];
        if (i >= k) continue;
        for (int s = v2n[i]; s >= 0 && s != kn; s = npar[s]) {
          if (flag[s] == k) break;
          flag[s] = k;
          T.contrib_rows[T.contrib_ptr[s] + fillc[s]++] = ka;
        }
      }
    }
  }
  if (P)
    for (int i = 0; i < n; i++) T.node_to_var[i] = P[T.node_to_var[i]];
  if (T.permuted) {
    T.invperm = iperm;
  } else {
    T.invperm.resize(n);
    std::iota(T.invperm.begin(), T.invperm.end(), 0);
  }
}

}  // namespace ab
