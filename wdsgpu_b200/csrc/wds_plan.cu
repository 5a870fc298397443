// Host planner: symbolic analysis of the junction graph and the device tables
// of one network (replaces GGASolver.__init__'s index build,
// dgga/solver.py:239-369, and symbolic.build_symbolic, dgga/symbolic.py:475).
//
//  * ordering: minimum degree on the elimination graph (ties broken by the
//    smallest junction row), or a caller-supplied permutation;
//  * elimination tree and the structure of L by merging children's column
//    structures; columns scheduled by elimination-tree level (leaves first);
//  * left-looking LDL^T task lists: one task per entry of L, each a list of
//    (L_ik, L_jk, 1/D_k) update triples in ascending k;
//  * deterministic gather maps for the assembly (per-junction incidence lists
//    in the reference's scatter order, per-pair link lists).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "wds_internal.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// Minimum-degree ordering on the explicit elimination graph.
std::vector<int> min_degree(int n, std::vector<std::vector<int>> adj) {
  std::vector<int> deg(n), order;
  order.reserve(n);
  std::vector<char> alive(n, 1);
  std::set<std::pair<int, int>> pq;
  for (int i = 0; i < n; ++i) {
    deg[i] = (int)adj[i].size();
    pq.insert({deg[i], i});
  }
  std::vector<int> merged;
  while (!pq.empty()) {
    int v = pq.begin()->second;
    pq.erase(pq.begin());
    alive[v] = 0;
    order.push_back(v);
    std::vector<int> nb;
    for (int u : adj[v])
      if (alive[u]) nb.push_back(u);
    for (int u : nb) {
      pq.erase({deg[u], u});
      merged.clear();
      std::set_union(adj[u].begin(), adj[u].end(), nb.begin(), nb.end(),
                     std::back_inserter(merged));
      std::vector<int> nu;
      nu.reserve(merged.size());
      for (int w : merged)
        if (w != u && alive[w]) nu.push_back(w);
      adj[u].swap(nu);
      deg[u] = (int)adj[u].size();
      pq.insert({deg[u], u});
    }
    adj[v].clear();
  }
  return order;
}

struct Blob {
  std::vector<unsigned char> bytes;
  template <class T>
  size_t add(const std::vector<T>& v) {
    size_t off = (bytes.size() + 255) / 256 * 256;
    bytes.resize(off + std::max<size_t>(v.size() * sizeof(T), 1));
    if (!v.empty()) std::memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
    return off;
  }
};

// Byte offsets of the per-scenario workspace of `B` scenarios (terminal
// factor and coefficients kept for the adjoint, scratch vectors, link flows,
// top-block inverses, large-network state, pump derivatives), each array
// 256-byte aligned.  One function for the plan's own workspace and for the
// fixed array of wds_forward_noalloc, so the two layouts cannot drift apart.
struct WorkOff {
  size_t W, P, dr, emh, hge, dke, act, scr, valid, lk, M, state, pump, dj, bytes;
};

WorkOff work_layout(const wds::DevNet& d, int nscr, size_t B, size_t state_bytes) {
  WorkOff o{};
  size_t bytes = 0;
  auto take = [&](size_t n) { size_t off = bytes; bytes += (n + 255) / 256 * 256; return off; };
  const size_t pc = (size_t)std::max(d.npcv, 1);
  o.W = take(B * d.nnzL * 8); o.P = take(B * d.L * 8); o.dr = take(B * d.L * 8);
  o.emh = take(B * d.Nj * 8); o.hge = take(B * d.Nj * 8); o.dke = take(B * d.Nj * 8);
  o.act = take(B * pc); o.scr = take(B * (size_t)nscr * d.Nj * 8); o.valid = take(B * 4);
  o.lk = take(B * 2 * d.L * 8); o.M = take(B * (size_t)std::max(d.nT * d.nT, 1) * 8);
  o.state = take(d.wide ? B * state_bytes : 0); o.pump = take(B * 3 * (size_t)d.npump * 8);
  o.dj = take(B * d.Nj * 8);
  o.bytes = bytes;
  return o;
}

// The workspace arrays at `base` laid out by work_layout.
wds::DevWork work_at(unsigned char* base, const WorkOff& o, const wds::DevNet& d, int nscr) {
  wds::DevWork w{};
  w.W = (double*)(base + o.W); w.P = (double*)(base + o.P); w.dr = (double*)(base + o.dr);
  w.emh = (double*)(base + o.emh); w.hge = (double*)(base + o.hge);
  w.dke = (double*)(base + o.dke); w.act = (int8_t*)(base + o.act);
  w.scr = (double*)(base + o.scr); w.valid = (int*)(base + o.valid);
  w.lk = (double*)(base + o.lk); w.M = (double*)(base + o.M);
  w.state = d.wide ? base + o.state : nullptr;
  w.dpump = (double*)(base + o.pump);
  w.dj = (double*)(base + o.dj);
  w.nscr = nscr;
  return w;
}

}  // namespace

struct WdsPlan {
  wds::DevNet dn{};
  wds::DevWork dw{};
  wds::HostSym sym;
  void* dtab = nullptr;
  void* dwork = nullptr;
  int max_batch = 0;
  int threads = 256;
  int groups = 1;
  size_t smem_fwd = 0, smem_adj = 0;
  int nnzA_lower = 0;
  bool have_state = false;
  int state_batch = 0;
  // changes with every call that rewrites the workspace (a forward, the
  // unrolled reverse pass), so that a caller holding a pending backward can
  // tell whether its kept state is still the plan's
  int64_t gen = 0;
};

extern "C" const char* wds_last_error(void) { return g_err.c_str(); }

extern "C" int wds_plan(const WdsNetwork* net, int32_t max_batch, WdsPlan** out) {
  using namespace wds;
  if (!net || !out || max_batch <= 0) return fail(WDS_E_ARG, "wds_plan: bad argument");
  *out = nullptr;
  const int N = net->n_nodes, L = net->n_links;
  if (N <= 0 || L <= 0) return fail(WDS_E_ARG, "wds_plan: empty network");
  // ---- junction rows (file order) and fixed nodes
  std::vector<int> jrow(N, -1), jnodes, fix_idx(N, -1), fnodes;
  for (int i = 0; i < N; ++i) {
    if (net->node_type[i] == 0) {
      jrow[i] = (int)jnodes.size();
      jnodes.push_back(i);
    } else {
      fix_idx[i] = (int)fnodes.size();
      fnodes.push_back(i);
    }
  }
  const int Nj = (int)jnodes.size(), Nf = (int)fnodes.size();
  if (Nj == 0) return fail(WDS_E_ARG, "wds_plan: no junctions");
  for (int k = 0; k < L; ++k) {
    int a = net->link_n1[k], b = net->link_n2[k];
    if (a < 0 || a >= N || b < 0 || b >= N)
      return fail(WDS_E_ARG, "wds_plan: link end out of range");
    int kd = net->link_kind[k];
    if (kd < WDS_KIND_PIPE || kd > WDS_KIND_PSV)
      return fail(WDS_E_UNSUPPORTED, "wds_plan: unsupported link kind");
  }
  // ---- junction graph
  std::vector<std::vector<int>> adj(Nj);
  for (int k = 0; k < L; ++k) {
    int a = jrow[net->link_n1[k]], b = jrow[net->link_n2[k]];
    if (a >= 0 && b >= 0 && a != b) {
      adj[a].push_back(b);
      adj[b].push_back(a);
    }
  }
  for (auto& v : adj) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  // ---- ordering
  std::vector<int> perm(Nj), iperm(Nj);
  if (net->perm) {
    std::vector<char> seen(Nj, 0);
    for (int p = 0; p < Nj; ++p) {
      int r = net->perm[p];
      if (r < 0 || r >= Nj || seen[r]) return fail(WDS_E_ARG, "wds_plan: perm is not a permutation");
      seen[r] = 1;
      perm[p] = r;
    }
  } else {
    perm = min_degree(Nj, adj);
  }
  for (int p = 0; p < Nj; ++p) iperm[perm[p]] = p;
  // ---- symbolic factorisation: struct(L_j) = A_{>j,j} U children \ {j}.
  // Two passes: the second renumbers the columns by elimination-tree level
  // (a topological order, so the factor is the same up to labels) so that
  // every level is a contiguous range of columns and of slots.
  std::vector<std::vector<int>> cstruct, children;
  std::vector<int> parent, level, mark, colptr, rowidx, levptr, levcol;
  int nlev = 0;
  for (int pass = 0; pass < 2; ++pass) {
    cstruct.assign(Nj, {}); children.assign(Nj, {});
    parent.assign(Nj, -1); level.assign(Nj, 0); mark.assign(Nj, -1);
    for (int j = 0; j < Nj; ++j) {
      std::vector<int>& s = cstruct[j];
      mark[j] = j;
      for (int u : adj[perm[j]]) {
        int i = iperm[u];
        if (i > j && mark[i] != j) {
          mark[i] = j;
          s.push_back(i);
        }
      }
      int lv = 0;
      for (int c : children[j]) {
        lv = std::max(lv, level[c] + 1);
        for (int i : cstruct[c])
          if (i != j && mark[i] != j) {
            mark[i] = j;
            s.push_back(i);
          }
      }
      level[j] = lv;
      std::sort(s.begin(), s.end());
      if (!s.empty()) {
        parent[j] = s[0];
        children[s[0]].push_back(j);
      }
    }
    colptr.assign(Nj + 1, 0); rowidx.clear();
    for (int j = 0; j < Nj; ++j) colptr[j + 1] = colptr[j] + 1 + (int)cstruct[j].size();
    const int nnzL = colptr[Nj];
    rowidx.resize(nnzL);
    for (int j = 0; j < Nj; ++j) {
      rowidx[colptr[j]] = j;
      for (size_t t = 0; t < cstruct[j].size(); ++t) rowidx[colptr[j] + 1 + t] = cstruct[j][t];
    }
    nlev = 0;
    for (int j = 0; j < Nj; ++j) nlev = std::max(nlev, level[j] + 1);
    levptr.assign(nlev + 1, 0); levcol.clear();
    for (int j = 0; j < Nj; ++j) levptr[level[j] + 1]++;
    for (int l = 0; l < nlev; ++l) levptr[l + 1] += levptr[l];
    levcol.resize(Nj);
    {
      std::vector<int> pos(levptr.begin(), levptr.end() - 1);
      for (int j = 0; j < Nj; ++j) levcol[pos[level[j]]++] = j;
    }
    if (pass == 0) {
      std::vector<int> p2(Nj);
      for (int t = 0; t < Nj; ++t) p2[t] = perm[levcol[t]];
      perm = p2;
      for (int p = 0; p < Nj; ++p) iperm[perm[p]] = p;
    }
  }
  const int nnzL = colptr[Nj];
  for (int t = 0; t < Nj; ++t)
    if (levcol[t] != t) return fail(WDS_E_ARG, "wds_plan: internal error (level order)");
  // ---- dense top block.  The top of the elimination tree is a thin chain
  // (many levels, few columns).  The columns of the top levels [L0, nlev), at
  // most WDS_TOP_MAX of them, are not factored column by column: their Schur
  // complement S (updates from the columns below only) is inverted densely,
  // and each substitution applies S^{-1} in one step instead of one step per
  // level in each sweep.  Worth it from three top levels on.
  if (net->top_max < -1 || net->top_max > WDS_TOP_MAX || net->groups_per_cta < 0 ||
      net->groups_per_cta > 4 || !(net->level_barrier_cost >= 0.0))
    return fail(WDS_E_ARG, "wds_plan: top_max must be -1..48, groups_per_cta 0..4, "
                           "level_barrier_cost >= 0");
  const int top_cap = net->top_max > 0 ? net->top_max : WDS_TOP_MAX;
  int L0 = nlev;
  for (int l = nlev - 1; l >= 0 && Nj - levptr[l] <= top_cap; --l) L0 = l;
  if (nlev - L0 < 3 || net->top_max < 0) L0 = nlev;
  const int cT = levptr[L0], nT = Nj - cT;
  auto slot = [&](int i, int j) -> int {  // slot of L_ij, i >= j; -1 if structurally zero
    if (i == j) return colptr[j];
    auto b = rowidx.begin() + colptr[j] + 1, e = rowidx.begin() + colptr[j + 1];
    auto it = std::lower_bound(b, e, i);
    if (it == e || *it != i) return -1;
    return (int)(it - rowidx.begin());
  };
  // row lists: rows[i] = { k < i : i in struct(k) } ascending; a top row keeps
  // only its entries in the columns below the top block
  std::vector<std::vector<int>> rows(Nj);
  for (int k = 0; k < Nj; ++k)
    for (int i : cstruct[k])
      if (i < cT || k < cT) rows[i].push_back(k);
  // forward-substitution items in level order: {j, first row entry, end, diag slot};
  // row entries {slot of L_jk, k} stored contiguously in the same order
  std::vector<int2> rent;
  std::vector<int4> fitem(Nj), bitem(Nj);
  for (int t = 0; t < Nj; ++t) {
    int j = levcol[t];
    int e0 = (int)rent.size();
    for (int k : rows[j]) rent.push_back(make_int2(slot(j, k), k));
    fitem[t] = make_int4(j, e0, (int)rent.size(), colptr[j]);
    bitem[t] = make_int4(j, colptr[j], colptr[j + 1], 0);
  }
  if (rent.empty()) rent.push_back(make_int2(0, 0));
  // factor tasks by level
  std::vector<int> ftask_ptr(nlev + 1, 0), fpair;
  std::vector<int4> ftask;
  for (int l = 0; l < nlev; ++l) {
    for (int t = levptr[l]; t < levptr[l + 1]; ++t) {
      int j = levcol[t];
      for (int e = colptr[j]; e < colptr[j + 1]; ++e) {
        int i = rowidx[e];
        int pb = (int)fpair.size() / 3;
        for (int k : rows[j]) {
          int sik = slot(i, k);
          if (sik < 0) continue;
          fpair.push_back(sik);
          fpair.push_back(slot(j, k));
          fpair.push_back(colptr[k]);
        }
        int pe = (int)fpair.size() / 3;
        ftask.push_back(make_int4(e, pb, pe, (i == j && j < cT) ? 1 : 0));
      }
    }
    ftask_ptr[l + 1] = (int)ftask.size();
  }
  // Execution mode per level and operation, one byte: bits 0-2 = log2 of the
  // lane-group size G (each item's dot product is spread over G lanes and
  // reduced with warp shuffles), bit 7 = wide (all 256 threads of the group,
  // followed by a group barrier) instead of narrow (warp 0 only, __syncwarp).
  // Cost model in units of one dependent round: rounds * (ceil(maxlen / G) +
  // 0.6 log2 G + 1), plus 0.5 per group barrier.
  const double bar_cost = net->level_barrier_cost > 0.0 ? net->level_barrier_cost : 0.5;
  auto pick_mode = [bar_cost](int count, int maxlen) -> uint8_t {
    double best = 1e30;
    uint8_t mode = 0;
    for (int wide = 0; wide <= 1; ++wide)
      for (int lg = 0; lg <= 5; ++lg) {
        const int G = 1 << lg, per = (wide ? 256 : 32) / G;
        const double rounds = (double)((count + per - 1) / per);
        const double cost =
            rounds * ((maxlen + G - 1) / G + 0.6 * lg + 1.0) + (wide ? bar_cost : 0.0);
        if (cost < best - 1e-12) { best = cost; mode = (uint8_t)(lg | (wide ? 0x80 : 0)); }
      }
    return mode;
  };
  // Level L0 (when the top block exists) stands for all top levels: its
  // factor mode is that of the Schur-complement step over every top slot, its
  // forward mode that of the step that subtracts the lower columns from the
  // top rows.
  std::vector<uint8_t> md_fac(nlev), md_fwd(nlev), md_bwd(nlev);
  for (int l = 0; l < nlev; ++l) {
    const int l1 = l == L0 ? nlev : l + 1;
    int mf = 0, mr = 0, mc = 0;
    for (int t = ftask_ptr[l]; t < ftask_ptr[l1]; ++t) mf = std::max(mf, ftask[t].z - ftask[t].y);
    for (int t = levptr[l]; t < levptr[l1]; ++t) {
      int j = levcol[t];
      mr = std::max(mr, (int)rows[j].size());
      mc = std::max(mc, colptr[j + 1] - colptr[j] - 1);
    }
    md_fac[l] = pick_mode(ftask_ptr[l1] - ftask_ptr[l], mf);
    md_fwd[l] = pick_mode(levptr[l1] - levptr[l], mr);
    md_bwd[l] = pick_mode(levptr[l1] - levptr[l], mc);
    if (l1 == nlev) break;
  }
  // dense position (i, j), i >= j, of the top block -> slot of L, or -1
  std::vector<int> dsl((size_t)std::max(nT * (nT + 1) / 2, 1), -1);
  for (int i = 0; i < nT; ++i)
    for (int j = 0; j <= i; ++j) dsl[(size_t)i * (i + 1) / 2 + j] = slot(cT + i, cT + j);
  // ---- link end codes, incidence lists, pairs
  auto code = [&](int nd) { return jrow[nd] >= 0 ? iperm[jrow[nd]] : -(fix_idx[nd] + 1); };
  std::vector<int> e1(L), e2(L);
  for (int k = 0; k < L; ++k) {
    e1[k] = code(net->link_n1[k]);
    e2[k] = code(net->link_n2[k]);
  }
  std::vector<std::vector<int>> inc1(Nj), inc2(Nj), finc1(Nf), finc2(Nf);
  for (int k = 0; k < L; ++k) {
    if (e1[k] >= 0) inc1[e1[k]].push_back(k); else finc1[-e1[k] - 1].push_back(k);
    if (e2[k] >= 0) inc2[e2[k]].push_back(k); else finc2[-e2[k] - 1].push_back(k);
  }
  std::vector<int> inc_ptr(Nj + 1, 0), inc_split(Nj), inc;
  for (int p = 0; p < Nj; ++p) {
    inc.insert(inc.end(), inc1[p].begin(), inc1[p].end());
    inc_split[p] = (int)inc.size();
    inc.insert(inc.end(), inc2[p].begin(), inc2[p].end());
    inc_ptr[p + 1] = (int)inc.size();
  }
  std::vector<int> finc_ptr(Nf + 1, 0), finc_split(std::max(Nf, 1), 0), finc;
  for (int f = 0; f < Nf; ++f) {
    finc.insert(finc.end(), finc1[f].begin(), finc1[f].end());
    finc_split[f] = (int)finc.size();
    finc.insert(finc.end(), finc2[f].begin(), finc2[f].end());
    finc_ptr[f + 1] = (int)finc.size();
  }
  std::map<std::pair<int, int>, std::vector<int>> pairs;
  for (int k = 0; k < L; ++k)
    if (e1[k] >= 0 && e2[k] >= 0 && e1[k] != e2[k])
      pairs[{std::max(e1[k], e2[k]), std::min(e1[k], e2[k])}].push_back(k);
  std::vector<int> pair_ptr(1, 0), pair_link, pair_slot;
  std::vector<char> is_a(nnzL, 0);
  std::map<std::pair<int, int>, int> pair_slot_of;
  for (auto& kv : pairs) {
    int s = slot(kv.first.first, kv.first.second);
    if (s < 0) return fail(WDS_E_ARG, "wds_plan: internal error (pair outside pattern)");
    is_a[s] = 1;
    pair_slot_of[kv.first] = s;
    pair_slot.push_back(s);
    pair_link.insert(pair_link.end(), kv.second.begin(), kv.second.end());
    pair_ptr.push_back((int)pair_link.size());
  }
  std::vector<int> fill_slot;
  for (int j = 0; j < Nj; ++j)
    for (int e = colptr[j] + 1; e < colptr[j + 1]; ++e)
      if (!is_a[e]) fill_slot.push_back(e);
  // ---- status-machine PRVs
  // (PRVs and PSVs with a setting, in link order)
  std::vector<int> link_pcv(L, -1), pcv_link, pcv_j1, pcv_j2, pcv_off, pcv_xf, node_xf(Nj, -1);
  std::vector<int> pcv_jc, pcv_jo, pcv_psv;
  std::vector<double> pcv_hset, pcv_km, pcv_sgn;
  int nxf = 0;
  for (int k = 0; k < L; ++k) {
    const bool psv = net->link_kind[k] == WDS_KIND_PSV;
    if (net->link_kind[k] != WDS_KIND_PRV && !psv) continue;
    if (e1[k] < 0 || e2[k] < 0)
      return fail(WDS_E_UNSUPPORTED,
                  "wds_plan: a PRV or PSV with a setting must join two junctions");
    const int jc = psv ? e1[k] : e2[k], jo = psv ? e2[k] : e1[k];
    link_pcv[k] = (int)pcv_link.size();
    pcv_link.push_back(k);
    pcv_j1.push_back(e1[k]);
    pcv_j2.push_back(e2[k]);
    pcv_jc.push_back(jc);
    pcv_jo.push_back(jo);
    pcv_sgn.push_back(psv ? -1.0 : 1.0);
    pcv_psv.push_back(psv ? 1 : 0);
    pcv_off.push_back(pair_slot_of[{std::max(e1[k], e2[k]), std::min(e1[k], e2[k])}]);
    if (node_xf[jc] < 0) node_xf[jc] = nxf++;
    pcv_xf.push_back(node_xf[jc]);
    pcv_hset.push_back(net->prv_hset[k]);
    pcv_km.push_back(net->km[k]);
  }
  const int npcv = (int)pcv_link.size();
  // ---- status-machine FCVs, and the valve pass order (link order)
  std::vector<int> link_fcv(L, -1), fcv_link, fcv_j1, fcv_j2, fcv_off, fcv_xf1, fcv_xf2, vord;
  std::vector<double> fcv_qs, fcv_km;
  for (int k = 0; k < L; ++k) {
    if (link_pcv[k] >= 0) vord.push_back(link_pcv[k]);
    if (net->link_kind[k] != WDS_KIND_FCV) continue;
    if (e1[k] < 0 || e2[k] < 0)
      return fail(WDS_E_UNSUPPORTED, "wds_plan: an FCV with a setting must join two junctions");
    link_fcv[k] = (int)fcv_link.size();
    vord.push_back(-1 - (int)fcv_link.size());
    fcv_link.push_back(k);
    fcv_j1.push_back(e1[k]);
    fcv_j2.push_back(e2[k]);
    fcv_off.push_back(pair_slot_of[{std::max(e1[k], e2[k]), std::min(e1[k], e2[k])}]);
    fcv_xf1.push_back(node_xf[e1[k]]);
    fcv_xf2.push_back(node_xf[e2[k]]);
    fcv_qs.push_back(net->prv_hset[k]);
    fcv_km.push_back(net->km[k]);
  }
  const int nfcv = (int)fcv_link.size();
  std::vector<int> cb_ptr(Nj + 1, 0), cb_idx;
  {
    std::vector<std::vector<int>> cb(Nj);
    for (int i = 0; i < npcv; ++i) cb[pcv_jc[i]].push_back(i);
    for (int p = 0; p < Nj; ++p) {
      cb_idx.insert(cb_idx.end(), cb[p].begin(), cb[p].end());
      cb_ptr[p + 1] = (int)cb_idx.size();
    }
  }
  // ---- tank links
  const int ntl = net->n_tank_links;
  std::vector<int> link_tl(L, -1), tl_link(ntl), tl_tank(ntl), tl_other(ntl);
  std::vector<double> tl_qsign(ntl), tl_hmax(ntl), tl_hmin(ntl);
  std::vector<uint8_t> tl_flags(ntl);
  for (int t = 0; t < ntl; ++t) {
    int k = net->tl_link[t];
    if (k < 0 || k >= L || fix_idx[net->tl_tank[t]] < 0)
      return fail(WDS_E_ARG, "wds_plan: bad tank link");
    link_tl[k] = t;
    tl_link[t] = k;
    tl_tank[t] = fix_idx[net->tl_tank[t]];
    tl_other[t] = code(net->tl_other[t]);
    tl_qsign[t] = net->tl_qsign[t];
    tl_hmax[t] = net->tl_hmax[t];
    tl_hmin[t] = net->tl_hmin[t];
    tl_flags[t] = net->tl_flags[t];
  }
  // ---- per-link copies
  std::vector<int8_t> kind(net->link_kind, net->link_kind + L),
      st0(net->status0, net->status0 + L), ptype(net->pump_type, net->pump_type + L);
  std::vector<uint8_t> flags(net->link_flags, net->link_flags + L);
  std::vector<double> km(net->km, net->km + L), km_tcv(net->km_tcv, net->km_tcv + L),
      q_init(net->q_init, net->q_init + L), ph0(net->pump_h0, net->pump_h0 + L),
      pr(net->pump_r, net->pump_r + L), pn(net->pump_n, net->pump_n + L),
      psp(net->pump_speed, net->pump_speed + L), phm(net->pump_hmax, net->pump_hmax + L);
  // pump index of each link, and the pumpstatus shut-off head at unit speed
  // (used when a call passes its own speeds)
  std::vector<int> link_pump(L, -1);
  std::vector<double> phu(L, 0.0);
  int npump = 0;
  for (int k = 0; k < L; ++k) {
    if (kind[k] != WDS_KIND_PUMP) continue;
    link_pump[k] = npump++;
    if (net->pump_hunit)
      phu[k] = net->pump_hunit[k];
    else
      phu[k] = psp[k] != 0.0 ? phm[k] / (psp[k] * psp[k]) : 0.0;
  }
  std::vector<int> cptr(net->curve_ptr, net->curve_ptr + L + 1);
  std::vector<double> cx(net->curve_x, net->curve_x + cptr[L]), cy(net->curve_y, net->curve_y + cptr[L]);
  std::vector<double> el(Nj);
  std::vector<int> jn(Nj);
  for (int p = 0; p < Nj; ++p) {
    jn[p] = jnodes[perm[p]];
    el[p] = net->elev[jn[p]];
  }
  // ---- bounds check of every index the kernels dereference (host side, so
  // that a table error is an error return and never a device fault)
  {
    auto in = [](int v, int lo, int hi) { return v >= lo && v < hi; };
    auto endok = [&](int c) { return c >= 0 ? c < Nj : (-c - 1) < Nf; };
    bool ok = true;
    for (int k = 0; k < L && ok; ++k) ok = endok(e1[k]) && endok(e2[k]);
    for (int v : inc) ok = ok && in(v, 0, L);
    for (int v : finc) ok = ok && in(v, 0, L);
    for (int v : pair_link) ok = ok && in(v, 0, L);
    for (int v : pair_slot) ok = ok && in(v, 0, nnzL);
    for (int v : fill_slot) ok = ok && in(v, 0, nnzL);
    for (int v : rowidx) ok = ok && in(v, 0, Nj);
    for (int v : levcol) ok = ok && in(v, 0, Nj);
    for (int v : fpair) ok = ok && in(v, 0, nnzL);
    for (auto& t : ftask) ok = ok && in(t.x, 0, nnzL) && t.y >= 0 && t.y <= t.z &&
                             t.z <= (int)fpair.size() / 3;
    for (auto& r : rent) ok = ok && in(r.x, 0, nnzL) && in(r.y, 0, Nj);
    for (int t = 0; t < Nj; ++t)
      ok = ok && in(fitem[t].x, 0, Nj) && fitem[t].y >= 0 && fitem[t].y <= fitem[t].z &&
           fitem[t].z <= (int)rent.size() && in(fitem[t].w, 0, nnzL) && in(bitem[t].x, 0, Nj) &&
           bitem[t].y >= 0 && bitem[t].y < bitem[t].z && bitem[t].z <= nnzL;
    for (int v : dsl) ok = ok && (v == -1 || in(v, colptr[cT], nnzL));
    ok = ok && nT >= 0 && nT <= WDS_TOP_MAX;
    for (int v : cb_idx) ok = ok && in(v, 0, std::max(npcv, 1));
    for (int i = 0; i < npcv; ++i)
      ok = ok && in(pcv_j1[i], 0, Nj) && in(pcv_j2[i], 0, Nj) && in(pcv_off[i], 0, nnzL) &&
           in(pcv_xf[i], 0, std::max(nxf, 1)) && in(pcv_link[i], 0, L) &&
           in(pcv_jc[i], 0, Nj) && in(pcv_jo[i], 0, Nj);
    for (int f = 0; f < nfcv; ++f)
      ok = ok && in(fcv_j1[f], 0, Nj) && in(fcv_j2[f], 0, Nj) && in(fcv_off[f], 0, nnzL) &&
           in(fcv_xf1[f], -1, std::max(nxf, 1)) && in(fcv_xf2[f], -1, std::max(nxf, 1)) &&
           in(fcv_link[f], 0, L);
    ok = ok && (int)vord.size() == npcv + nfcv;
    for (int v : vord) ok = ok && (v >= 0 ? v < npcv : (-1 - v) < nfcv);
    for (int p = 0; p < Nj; ++p) ok = ok && node_xf[p] < std::max(nxf, 1);
    for (int t = 0; t < ntl; ++t) ok = ok && in(tl_tank[t], 0, Nf) && endok(tl_other[t]);
    for (int k = 0; k < L; ++k) {
      if (net->pump_type[k] == 2 && net->link_kind[k] == WDS_KIND_PUMP)
        ok = ok && net->curve_ptr[k + 1] - net->curve_ptr[k] >= 2;
      ok = ok && net->curve_ptr[k] <= net->curve_ptr[k + 1];
    }
    for (int p = 0; p < Nj; ++p) ok = ok && in(jn[p], 0, N);
    for (int f = 0; f < Nf; ++f) ok = ok && in(fnodes[f], 0, N);
    if (!ok) return fail(WDS_E_ARG, "wds_plan: internal table failed its bounds check");
  }
  // ---- compact tables.  Junction, link and incidence indices are 16-bit.
  // Slot-valued tables (positions in W, in the update-term list, in the row
  // lists) are 16-bit and staged in shared memory when the network allows it
  // (narrow layout); otherwise they are 32-bit and read from global memory,
  // with the scenario state there too (wide layout, large networks).
  if (Nj >= 32768 || Nf >= 16384 || L >= 32768 || N >= 65536 || (int)inc.size() >= 65536 ||
      (int)pair_link.size() >= 65536)
    return fail(WDS_E_UNSUPPORTED, "wds_plan: network too large (at most 32767 junctions and "
                                   "32767 links)");
  for (auto& t : ftask)
    if (t.z - t.y >= 32768) return fail(WDS_E_UNSUPPORTED, "wds_plan: update list too long");
  // Columns are numbered in level order, so level l owns the columns
  // [levptr[l], levptr[l+1]) and the slots [colptr[levptr[l]], colptr[levptr[l+1]]).
  for (int j = 0; j < Nj; ++j)
    if (fitem[j].x != j || (j > 0 && fitem[j].y != fitem[j - 1].z) || (j == 0 && fitem[0].y != 0))
      return fail(WDS_E_ARG, "wds_plan: internal error (row list order)");
  std::vector<uint16_t> s_ri(rowidx.begin(), rowidx.end());
  std::vector<uint16_t> s_lp(levptr.begin(), levptr.end());
  std::vector<uint8_t> s_md;
  s_md.insert(s_md.end(), md_fac.begin(), md_fac.end());
  s_md.insert(s_md.end(), md_fwd.begin(), md_fwd.end());
  s_md.insert(s_md.end(), md_bwd.begin(), md_bwd.end());
  // incidence entries: link | PRV-with-setting << 16 | other end fixed << 17 | fixed index << 18
  std::vector<uint16_t> s_ip(inc_ptr.begin(), inc_ptr.end()), s_is(inc_split.begin(), inc_split.end());
  std::vector<uint32_t> s_in(inc.size());
  for (int p = 0; p < Nj; ++p)
    for (int e = inc_ptr[p]; e < inc_ptr[p + 1]; ++e) {
      const int k = inc[e];
      const int other = e < inc_split[p] ? e2[k] : e1[k];
      uint32_t v = (uint32_t)k;
      if (net->link_kind[k] == WDS_KIND_PRV || net->link_kind[k] == WDS_KIND_FCV ||
          net->link_kind[k] == WDS_KIND_PSV)
        v |= 1u << 16;
      if (other < 0) v |= (1u << 17) | ((uint32_t)(-other - 1) << 18);
      s_in[e] = v;
    }
  if (s_in.empty()) s_in.push_back(0);
  std::vector<int16_t> s_e1(e1.begin(), e1.end()), s_e2(e2.begin(), e2.end());
  std::vector<uint16_t> s_pp(pair_ptr.begin(), pair_ptr.end());
  std::vector<uint16_t> s_pl(pair_link.size());
  for (size_t e = 0; e < pair_link.size(); ++e)
    s_pl[e] = (uint16_t)(pair_link[e] | ((net->link_kind[pair_link[e]] == WDS_KIND_PRV ||
                                          net->link_kind[pair_link[e]] == WDS_KIND_FCV ||
                                          net->link_kind[pair_link[e]] == WDS_KIND_PSV) ? 0x8000 : 0));
  if (s_pl.empty()) s_pl.push_back(0);
  struct TabOff { int sp, fp, cp, ri, lp, rp, re, md, ip, is, in, e1, e2, pp, pl, ps, fl, ds; };
  auto pack = [&](auto tag, Blob& sb, TabOff& o) {
    using S = decltype(tag);
    constexpr bool W32 = sizeof(S) == 4;
    auto sadd = [&](auto& v) {
      size_t off = (sb.bytes.size() + 15) / 16 * 16;
      size_t nb = v.size() * sizeof(v[0]);
      sb.bytes.resize(off + nb);
      if (nb) std::memcpy(sb.bytes.data() + off, v.data(), nb);
      return (int)off;
    };
    // update list of every entry of L, by slot (narrow: begin | count << 16 |
    // diagonal << 31; wide: begin, count | diagonal << 31)
    std::vector<uint32_t> sp((size_t)nnzL * (W32 ? 2 : 1), 0);
    for (auto& t : ftask) {
      const uint32_t hi = (uint32_t)(t.z - t.y) | ((uint32_t)t.w << 31);
      if (W32) { sp[2 * (size_t)t.x] = (uint32_t)t.y; sp[2 * (size_t)t.x + 1] = hi; }
      else sp[t.x] = (uint32_t)t.y | ((uint32_t)(t.z - t.y) << 16) | ((uint32_t)t.w << 31);
    }
    std::vector<S> fp(fpair.begin(), fpair.end());
    if (fp.empty()) fp.push_back(0);
    std::vector<S> cp(colptr.begin(), colptr.end());
    // row lists (forward substitution): entries {slot of L_jk, k} of row j at [rptr[j], rptr[j+1])
    std::vector<S> rp(Nj + 1, 0);
    for (int j = 0; j < Nj; ++j) rp[j + 1] = (S)fitem[j].z;
    std::vector<uint32_t> re(rent.size() * (W32 ? 2 : 1));
    for (size_t e = 0; e < rent.size(); ++e) {
      if (W32) { re[2 * e] = (uint32_t)rent[e].x; re[2 * e + 1] = (uint32_t)rent[e].y; }
      else re[e] = (uint32_t)rent[e].x | ((uint32_t)rent[e].y << 16);
    }
    std::vector<S> ps(pair_slot.begin(), pair_slot.end());
    if (ps.empty()) ps.push_back(0);
    std::vector<S> fl(fill_slot.begin(), fill_slot.end());
    if (fl.empty()) fl.push_back(0);
    std::vector<S> ds(dsl.size());
    for (size_t i = 0; i < dsl.size(); ++i) ds[i] = dsl[i] < 0 ? (S)~S(0) : (S)dsl[i];
    o.sp = sadd(sp); o.fp = sadd(fp); o.cp = sadd(cp); o.ri = sadd(s_ri); o.lp = sadd(s_lp);
    o.rp = sadd(rp); o.re = sadd(re); o.md = sadd(s_md); o.ip = sadd(s_ip); o.is = sadd(s_is);
    o.in = sadd(s_in); o.e1 = sadd(s_e1); o.e2 = sadd(s_e2); o.pp = sadd(s_pp); o.pl = sadd(s_pl);
    o.ps = sadd(ps); o.fl = sadd(fl); o.ds = sadd(ds);
    sb.bytes.resize((sb.bytes.size() + 15) / 16 * 16);
  };
  const bool fits16 = nnzL < 65535 && (int)fpair.size() / 3 < 65536 &&
                      (int)rent.size() < 65536 && (int)fitem.back().z < 65536;
  // per-scenario state of the shared-memory layout (sizes only)
  DevNet dsz{};
  dsz.N = N; dsz.L = L; dsz.Nj = Nj; dsz.Nf = Nf; dsz.nnzL = nnzL; dsz.npcv = npcv;
  dsz.nxf = nxf; dsz.nT = nT;
  dsz.emcap = std::min(Nj, net->emitter_capacity > 0 ? net->emitter_capacity : 64);
  dsz.fp32 = net->factor_fp32 ? 1 : 0;
  const size_t state_bytes = state_smem_bytes(dsz);
  Blob sblob;
  TabOff to{};
  if (net->layout < WDS_LAYOUT_AUTO || net->layout > WDS_LAYOUT_GLOBAL)
    return fail(WDS_E_ARG, "wds_plan: unknown layout");
  bool wide = !fits16 || net->layout == WDS_LAYOUT_GLOBAL;
  if (!wide) {
    pack(uint16_t{}, sblob, to);
    wide = sblob.bytes.size() + state_bytes > 227 * 1024;
  }
  if (wide && net->layout == WDS_LAYOUT_SHARED)
    return fail(WDS_E_UNSUPPORTED, "wds_plan: the network's tables and state exceed shared "
                                   "memory (layout WDS_LAYOUT_SHARED)");
  if (wide) {
    sblob = Blob();
    pack(uint32_t{}, sblob, to);
  }
  std::vector<unsigned char> stab_bytes = sblob.bytes;
  // ---- upload
  Blob blob;
  size_t o_e1 = blob.add(e1), o_e2 = blob.add(e2), o_kind = blob.add(kind), o_flags = blob.add(flags),
         o_st0 = blob.add(st0), o_ptype = blob.add(ptype), o_km = blob.add(km),
         o_kmt = blob.add(km_tcv), o_q0 = blob.add(q_init), o_ph0 = blob.add(ph0),
         o_pr = blob.add(pr), o_pn = blob.add(pn), o_psp = blob.add(psp), o_phm = blob.add(phm),
         o_cptr = blob.add(cptr), o_cx = blob.add(cx), o_cy = blob.add(cy),
         o_ltl = blob.add(link_tl), o_lpcv = blob.add(link_pcv), o_jn = blob.add(jn),
         o_el = blob.add(el), o_incp = blob.add(inc_ptr), o_incs = blob.add(inc_split),
         o_inc = blob.add(inc), o_nxf = blob.add(node_xf), o_cbp = blob.add(cb_ptr),
         o_cbi = blob.add(cb_idx), o_fn = blob.add(fnodes), o_fincp = blob.add(finc_ptr),
         o_fincs = blob.add(finc_split), o_finc = blob.add(finc), o_pp = blob.add(pair_ptr),
         o_pl = blob.add(pair_link), o_ps = blob.add(pair_slot), o_fs = blob.add(fill_slot),
         o_cp = blob.add(colptr), o_ri = blob.add(rowidx), o_lp = blob.add(levptr),
         o_lc = blob.add(levcol), o_ftp = blob.add(ftask_ptr), o_ft = blob.add(ftask),
         o_fp = blob.add(fpair), o_rent = blob.add(rent), o_fit = blob.add(fitem),
         o_bit = blob.add(bitem),
         o_pcl = blob.add(pcv_link), o_pj1 = blob.add(pcv_j1), o_pj2 = blob.add(pcv_j2),
         o_poff = blob.add(pcv_off), o_pxf = blob.add(pcv_xf), o_phs = blob.add(pcv_hset),
         o_pkm = blob.add(pcv_km), o_tll = blob.add(tl_link), o_tlt = blob.add(tl_tank),
         o_tlo = blob.add(tl_other), o_tlq = blob.add(tl_qsign), o_tlx = blob.add(tl_hmax),
         o_tln = blob.add(tl_hmin), o_tlf = blob.add(tl_flags), o_stab = blob.add(stab_bytes),
         o_lpu = blob.add(link_pump), o_phu = blob.add(phu), o_lfc = blob.add(link_fcv),
         o_fcl = blob.add(fcv_link), o_fj1 = blob.add(fcv_j1), o_fj2 = blob.add(fcv_j2),
         o_fof = blob.add(fcv_off), o_fx1 = blob.add(fcv_xf1), o_fx2 = blob.add(fcv_xf2),
         o_fqs = blob.add(fcv_qs), o_fkm = blob.add(fcv_km), o_vord = blob.add(vord),
         o_pjc = blob.add(pcv_jc), o_pjo = blob.add(pcv_jo), o_psg = blob.add(pcv_sgn),
         o_pps = blob.add(pcv_psv);
  WdsPlan* plan = new WdsPlan();
  if (cudaMalloc(&plan->dtab, blob.bytes.size()) != cudaSuccess) {
    delete plan;
    return fail(WDS_E_NOMEM, "wds_plan: cudaMalloc of the device tables failed");
  }
  if (cudaMemcpy(plan->dtab, blob.bytes.data(), blob.bytes.size(), cudaMemcpyHostToDevice) !=
      cudaSuccess) {
    cudaFree(plan->dtab);
    delete plan;
    return fail(WDS_E_CUDA, "wds_plan: upload of the device tables failed");
  }
  unsigned char* base = (unsigned char*)plan->dtab;
#define P_(T, off) reinterpret_cast<const T*>(base + (off))
  DevNet& d = plan->dn;
  d.N = N; d.L = L; d.Nj = Nj; d.Nf = Nf; d.nnzL = nnzL; d.nlev = nlev; d.npcv = npcv;
  d.ntl = ntl; d.npairs = (int)pair_slot.size(); d.nfill = (int)fill_slot.size(); d.nxf = nxf;
  d.nftask = (int)ftask.size(); d.nfpair = (int)fpair.size() / 3;
  d.e1 = P_(int, o_e1); d.e2 = P_(int, o_e2); d.kind = P_(int8_t, o_kind);
  d.flags = P_(uint8_t, o_flags); d.status0 = P_(int8_t, o_st0); d.ptype = P_(int8_t, o_ptype);
  d.km = P_(double, o_km); d.km_tcv = P_(double, o_kmt); d.q_init = P_(double, o_q0);
  d.ph0 = P_(double, o_ph0); d.pr = P_(double, o_pr); d.pn = P_(double, o_pn);
  d.pspeed = P_(double, o_psp); d.phmax = P_(double, o_phm); d.cptr = P_(int, o_cptr);
  d.phunit = P_(double, o_phu); d.link_pump = P_(int, o_lpu); d.npump = npump;
  d.nfcv = nfcv; d.link_fcv = P_(int, o_lfc); d.fcv_link = P_(int, o_fcl);
  d.fcv_j1 = P_(int, o_fj1); d.fcv_j2 = P_(int, o_fj2); d.fcv_off = P_(int, o_fof);
  d.fcv_xf1 = P_(int, o_fx1); d.fcv_xf2 = P_(int, o_fx2); d.fcv_qs = P_(double, o_fqs);
  d.fcv_km = P_(double, o_fkm); d.vord = P_(int, o_vord);
  d.pcv_jc = P_(int, o_pjc); d.pcv_jo = P_(int, o_pjo); d.pcv_sgn = P_(double, o_psg);
  d.pcv_psv = P_(int, o_pps);
  d.cx = P_(double, o_cx); d.cy = P_(double, o_cy); d.link_tl = P_(int, o_ltl);
  d.link_pcv = P_(int, o_lpcv); d.jnode = P_(int, o_jn); d.el = P_(double, o_el);
  d.inc_ptr = P_(int, o_incp); d.inc_split = P_(int, o_incs); d.inc = P_(int, o_inc);
  d.node_xf = P_(int, o_nxf); d.cb_ptr = P_(int, o_cbp); d.cb_idx = P_(int, o_cbi);
  d.fnode = P_(int, o_fn); d.finc_ptr = P_(int, o_fincp); d.finc_split = P_(int, o_fincs);
  d.finc = P_(int, o_finc); d.pair_ptr = P_(int, o_pp); d.pair_link = P_(int, o_pl);
  d.pair_slot = P_(int, o_ps); d.fill_slot = P_(int, o_fs); d.colptr = P_(int, o_cp);
  d.rowidx = P_(int, o_ri); d.levptr = P_(int, o_lp); d.levcol = P_(int, o_lc);
  d.ftask_ptr = P_(int, o_ftp); d.ftask = P_(int4, o_ft); d.fpair = P_(int, o_fp);
  d.rent = P_(int2, o_rent); d.fitem = P_(int4, o_fit); d.bitem = P_(int4, o_bit);
  d.pcv_link = P_(int, o_pcl); d.pcv_j1 = P_(int, o_pj1); d.pcv_j2 = P_(int, o_pj2);
  d.pcv_off = P_(int, o_poff); d.pcv_xf = P_(int, o_pxf); d.pcv_hset = P_(double, o_phs);
  d.pcv_km = P_(double, o_pkm); d.tl_link = P_(int, o_tll); d.tl_tank = P_(int, o_tlt);
  d.tl_other = P_(int, o_tlo); d.tl_qsign = P_(double, o_tlq); d.tl_hmax = P_(double, o_tlx);
  d.tl_hmin = P_(double, o_tln); d.tl_flags = P_(uint8_t, o_tlf);
  d.stab = P_(uint4, o_stab);
  d.wide = wide ? 1 : 0;
  d.fp32 = net->factor_fp32 ? 1 : 0;
  d.stab_bytes = wide ? 0 : (int)stab_bytes.size();  // staged into shared memory (narrow only)
  d.o_spair = to.sp; d.o_fpair = to.fp; d.o_colptr = to.cp;
  d.o_rowidx = to.ri; d.o_levptr = to.lp; d.o_rptr = to.rp;
  d.o_rent = to.re; d.o_mode = to.md; d.o_inc_ptr = to.ip; d.o_inc_split = to.is;
  d.o_inc = to.in; d.o_e1 = to.e1; d.o_e2 = to.e2; d.o_pptr = to.pp; d.o_plink = to.pl;
  d.o_pslot = to.ps; d.o_fill = to.fl; d.o_dslot = to.ds;
  d.L0 = L0; d.cT = cT; d.nT = nT;
#undef P_
  d.hexp = net->hexp; d.qexp = net->qexp; d.rqtol = net->rqtol; d.htol = net->htol;
  d.qtol = net->qtol; d.ucf_flow = net->ucf_flow; d.ucf_head = net->ucf_head;
  d.checkfreq = net->checkfreq; d.maxcheck = net->maxcheck; d.extra_iter = net->extra_iter;
  d.emcap = std::min(Nj, net->emitter_capacity > 0 ? net->emitter_capacity : 64);
  plan->nnzA_lower = Nj + (int)pair_slot.size();
  plan->threads = 256;
  // scenario groups per CTA: the count that keeps the most scenarios resident
  // per SM (228 KB of shared memory per SM, 1 KB reserved per CTA)
  if (d.wide) {  // large network: one 256-thread CTA per scenario, state in global memory
    plan->groups = 1;
    plan->smem_fwd = plan->smem_adj = 0;
  } else {
    const size_t st = state_smem_bytes(d);
    int best_g = 0, best_res = 0;
    for (int g = 1; g <= 4; ++g) {
      size_t sm = (size_t)d.stab_bytes + g * st;
      if (sm > 227 * 1024) break;
      int ctas = (int)((228 * 1024) / (sm + 1024));
      ctas = std::min(ctas, 2048 / (256 * g));
      if (ctas * g > best_res) { best_res = ctas * g; best_g = g; }
    }
    if (net->groups_per_cta > 0) {  // a tuned choice, if the state fits
      if ((size_t)d.stab_bytes + net->groups_per_cta * st > 227 * 1024) {
        cudaFree(plan->dtab);
        delete plan;
        return fail(WDS_E_ARG, "wds_plan: groups_per_cta " + std::to_string(net->groups_per_cta) +
                                   " exceeds shared memory for this network");
      }
      best_g = net->groups_per_cta;
    }
    plan->groups = best_g;
    plan->smem_fwd = best_g ? (size_t)d.stab_bytes + best_g * st : (size_t)d.stab_bytes + st;
    plan->smem_adj = plan->smem_fwd;
  }
  if (plan->groups == 0 || (!d.wide && plan->smem_fwd > 227 * 1024)) {
    cudaFree(plan->dtab);
    delete plan;
    return fail(WDS_E_UNSUPPORTED,
                "wds_plan: the network's per-scenario state exceeds shared memory");
  }
  // ---- workspace
  plan->max_batch = max_batch;
  DevWork& w = plan->dw;
  // heads, rp, res, sx, 2p Woodbury columns, 2p+1 per-warp temporaries
  const int nscr = 5 + 4 * std::max(npcv, 1);
  const WorkOff wo = work_layout(d, nscr, (size_t)max_batch, state_bytes);
  const size_t bytes = wo.bytes;
  if (cudaMalloc(&plan->dwork, bytes) != cudaSuccess) {
    cudaFree(plan->dtab);
    delete plan;
    return fail(WDS_E_NOMEM, "wds_plan: cudaMalloc of the workspace failed");
  }
  cudaMemset(plan->dwork, 0, bytes);
  w = work_at((unsigned char*)plan->dwork, wo, d, nscr);
  // ---- host copy of the symbolic structure
  HostSym& hs = plan->sym;
  hs.Nj = Nj; hs.perm = perm; hs.iperm = iperm; hs.parent = parent; hs.level = level;
  hs.colptr = colptr; hs.rowidx = rowidx;
  *out = plan;
  return WDS_OK;
}

extern "C" int wds_plan_stats(const WdsPlan* plan, int64_t* o) {
  if (!plan || !o) return fail(WDS_E_ARG, "wds_plan_stats: bad argument");
  o[0] = plan->dn.Nj; o[1] = plan->dn.nnzL; o[2] = plan->dn.nlev; o[3] = plan->dn.nfpair;
  o[4] = (int64_t)plan->smem_fwd; o[5] = plan->dn.npcv; o[6] = plan->nnzA_lower;
  o[7] = plan->groups;
  return WDS_OK;
}

extern "C" int wds_state_generation(const WdsPlan* plan, int64_t* gen) {
  if (!plan || !gen) return fail(WDS_E_ARG, "wds_state_generation: bad argument");
  *gen = plan->gen;
  return WDS_OK;
}

extern "C" int wds_plan_symbolic(const WdsPlan* plan, int32_t* perm, int32_t* colptr,
                                 int32_t* rowidx, int32_t* parent, int32_t* level) {
  if (!plan) return fail(WDS_E_ARG, "wds_plan_symbolic: bad argument");
  const auto& s = plan->sym;
  if (perm) std::copy(s.perm.begin(), s.perm.end(), perm);
  if (colptr) std::copy(s.colptr.begin(), s.colptr.end(), colptr);
  if (rowidx) std::copy(s.rowidx.begin(), s.rowidx.end(), rowidx);
  if (parent) std::copy(s.parent.begin(), s.parent.end(), parent);
  if (level) std::copy(s.level.begin(), s.level.end(), level);
  return WDS_OK;
}

namespace wds {
// Options of a forward call beyond the basic ones: pump parameters (rows of
// [L] at stride 0, one row for all scenarios, or L, one per scenario) and the
// refinement band of the GGA iterations.
static int set_pump_opts(FwdArgs& a, const WdsForwardOpts* o, int L, const std::string& who) {
  if (!(o->refine_band >= 0.0))
    return fail(WDS_E_ARG, who + ": refine_band must be >= 0");
  a.rband = o->refine_band;
  a.rec = o->unroll_record;
  a.diag = o->diag_ratio;
  a.sflags = o->sched_flags;
  a.schg = o->sched_chg;
  if ((a.sflags == nullptr) != (a.schg == nullptr))
    return fail(WDS_E_ARG, who + ": sched_flags and sched_chg go together");
  if (a.sflags && !o->status_machine)
    return fail(WDS_E_ARG, who + ": the schedule record needs status_machine 1");
  a.s0 = o->status0;
  if (a.rec && (o->status_machine || o->polish_steps >= 0))
    return fail(WDS_E_ARG, who + ": the unrolled mode runs with status_machine 0 and no polish");
  a.th_sp = o->pump_speed;
  a.th_h0 = o->pump_h0;
  a.th_r = o->pump_r;
  a.th_stride = o->pump_stride;
  if ((o->pump_speed || o->pump_h0 || o->pump_r) && o->pump_stride != 0 && o->pump_stride != L)
    return fail(WDS_E_ARG, who + ": pump_stride must be 0 or n_links");
  return WDS_OK;
}
}  // namespace wds

extern "C" int wds_forward(WdsPlan* plan, int32_t batch, const WdsForwardOpts* o,
                           const double* demand, const double* fixed_head, const double* ke,
                           const double* r, double* head, double* flow, double* emitter,
                           int8_t* status, int32_t* iters, double* relerr, int32_t* info,
                           void* stream) {
  using namespace wds;
  if (!plan || !o || batch <= 0) return fail(WDS_E_ARG, "wds_forward: bad argument");
  if (batch > plan->max_batch) return fail(WDS_E_ARG, "wds_forward: batch exceeds the plan's max_batch");
  if (!demand || !fixed_head || !ke || !r || !head || !flow || !emitter || !status || !iters ||
      !relerr || !info)
    return fail(WDS_E_ARG, "wds_forward: null pointer");
  if (o->max_iter <= 0 || !(o->accuracy > 0.0) || o->refine < 0)
    return fail(WDS_E_ARG, "wds_forward: bad options");
  FwdArgs a{};
  a.B = batch; a.hacc = o->accuracy; a.max_iter = o->max_iter; a.sm = o->status_machine ? 1 : 0;
  a.refine = o->refine; a.polish = o->polish_steps; a.ke_stride = o->ke_stride;
  a.r_stride = o->r_stride; a.d = demand; a.rh = fixed_head; a.ke = ke; a.r = r;
  a.q0 = o->q0; a.e0 = o->e0;
  if (int rc0 = set_pump_opts(a, o, plan->dn.L, "wds_forward"); rc0 != WDS_OK) return rc0;
  a.head = head; a.flow = flow; a.emit = emitter; a.status = status; a.iters = iters;
  a.relerr = relerr; a.info = info;
  std::string err;
  int rc = launch_forward(plan->dn, plan->dw, a, plan->groups, stream, &err);
  if (rc != WDS_OK) return fail(rc, err);
  plan->have_state = o->polish_steps >= 0;
  plan->state_batch = batch;
  ++plan->gen;
  return WDS_OK;
}

extern "C" int wds_adjoint_rhs(WdsPlan* plan, int32_t batch, int32_t rhs_per, int32_t first,
                               const double* gH, const double* gQ, const double* gE,
                               double* gd, double* grh, double* gke, double* gr,
                               void* stream) {
  using namespace wds;
  if (!plan || batch <= 0 || rhs_per <= 0 || first < 0 || !gH || !gQ || !gE || !gd || !grh ||
      !gke || !gr)
    return fail(WDS_E_ARG, "wds_adjoint_rhs: bad argument");
  if (batch > plan->max_batch)
    return fail(WDS_E_ARG, "wds_adjoint_rhs: batch exceeds the plan's max_batch");
  if (!plan->have_state)
    return fail(WDS_E_STATE, "wds_adjoint_rhs: no implicit forward to differentiate");
  if ((int64_t)first + batch - 1 >= (int64_t)plan->state_batch * rhs_per)
    return fail(WDS_E_ARG, "wds_adjoint_rhs: rows beyond the kept scenarios");
  AdjArgs a{batch, gH, gQ, gE, gd, grh, gke, gr};
  a.rhs_per = rhs_per;
  a.v0 = first;
  std::string err;
  int rc = launch_adjoint(plan->dn, plan->dw, a, plan->groups, stream, &err);
  if (rc != WDS_OK) return fail(rc, err);
  return WDS_OK;
}

extern "C" int wds_forward_multi(int32_t nplans, WdsPlan* const* plans, const int32_t* batch,
                                 const WdsForwardOpts* opts, const WdsForwardIO* io,
                                 void* stream) {
  using namespace wds;
  if (nplans <= 0 || nplans > WDS_MULTI_MAX || !plans || !batch || !opts || !io)
    return fail(WDS_E_ARG, "wds_forward_multi: bad argument (1 to 8 plans)");
  FwdJobs jobs{};
  jobs.n = nplans;
  for (int p = 0; p < nplans; ++p) {
    const WdsPlan* plan = plans[p];
    const WdsForwardOpts* o = &opts[p];
    const WdsForwardIO& x = io[p];
    if (!plan || batch[p] <= 0 || batch[p] > plan->max_batch)
      return fail(WDS_E_ARG, "wds_forward_multi: plan " + std::to_string(p) +
                                 ": bad plan or batch beyond its max_batch");
    if (!x.demand || !x.fixed_head || !x.ke || !x.r || !x.head || !x.flow || !x.emitter ||
        !x.status || !x.iters || !x.relerr || !x.info)
      return fail(WDS_E_ARG, "wds_forward_multi: plan " + std::to_string(p) + ": null pointer");
    if (o->max_iter <= 0 || !(o->accuracy > 0.0) || o->refine < 0)
      return fail(WDS_E_ARG, "wds_forward_multi: plan " + std::to_string(p) + ": bad options");
    for (int q = 0; q < p; ++q)
      if (plans[q] == plan)
        return fail(WDS_E_ARG, "wds_forward_multi: a plan appears twice (its workspace would be shared)");
    FwdJob& J = jobs.j[p];
    J.n = plan->dn;
    J.w = plan->dw;
    J.groups = plan->dn.wide ? 3 : std::min(3, plan->groups);
    FwdArgs& a = J.a;
    a.B = batch[p]; a.hacc = o->accuracy; a.max_iter = o->max_iter;
    a.sm = o->status_machine ? 1 : 0; a.refine = o->refine; a.polish = o->polish_steps;
    a.ke_stride = o->ke_stride; a.r_stride = o->r_stride;
    a.d = x.demand; a.rh = x.fixed_head; a.ke = x.ke; a.r = x.r; a.q0 = o->q0; a.e0 = o->e0;
    if (int rc0 = set_pump_opts(a, o, plan->dn.L, "wds_forward_multi: plan " + std::to_string(p));
        rc0 != WDS_OK)
      return rc0;
    a.head = x.head; a.flow = x.flow; a.emit = x.emitter; a.status = x.status;
    a.iters = x.iters; a.relerr = x.relerr; a.info = x.info;
  }
  std::string err;
  const int rc = launch_forward_multi(jobs, stream, &err);
  if (rc != WDS_OK) return fail(rc, err);
  for (int p = 0; p < nplans; ++p) {
    plans[p]->have_state = opts[p].polish_steps >= 0;
    plans[p]->state_batch = batch[p];
    ++plans[p]->gen;
  }
  return WDS_OK;
}

extern "C" int wds_adjoint_multi(int32_t nplans, WdsPlan* const* plans, const int32_t* batch,
                                 const WdsAdjointIO* io, void* stream) {
  using namespace wds;
  if (nplans <= 0 || nplans > WDS_MULTI_MAX || !plans || !batch || !io)
    return fail(WDS_E_ARG, "wds_adjoint_multi: bad argument (1 to 8 plans)");
  AdjJobs jobs{};
  jobs.n = nplans;
  for (int p = 0; p < nplans; ++p) {
    const WdsPlan* plan = plans[p];
    const WdsAdjointIO& x = io[p];
    if (!plan || batch[p] <= 0 || !x.gH || !x.gQ || !x.gE || !x.gd || !x.grh || !x.gke || !x.gr)
      return fail(WDS_E_ARG, "wds_adjoint_multi: plan " + std::to_string(p) + ": bad argument");
    if (!plan->have_state || batch[p] != plan->state_batch)
      return fail(WDS_E_STATE, "wds_adjoint_multi: plan " + std::to_string(p) +
                                   ": no implicit forward of this batch size to differentiate");
    AdjJob& J = jobs.j[p];
    J.n = plan->dn;
    J.w = plan->dw;
    J.groups = plan->dn.wide ? 3 : std::min(3, plan->groups);
    J.a = AdjArgs{batch[p], x.gH, x.gQ, x.gE, x.gd, x.grh, x.gke, x.gr};
  }
  std::string err;
  const int rc = launch_adjoint_multi(jobs, stream, &err);
  if (rc != WDS_OK) return fail(rc, err);
  return WDS_OK;
}

extern "C" int wds_adjoint(WdsPlan* plan, int32_t batch, const double* gH, const double* gQ,
                           const double* gE, double* gd, double* grh, double* gke, double* gr,
                           void* stream) {
  using namespace wds;
  if (!plan || batch <= 0 || !gH || !gQ || !gE || !gd || !grh || !gke || !gr)
    return fail(WDS_E_ARG, "wds_adjoint: bad argument");
  if (!plan->have_state || batch != plan->state_batch)
    return fail(WDS_E_STATE, "wds_adjoint: no implicit forward of this batch size to differentiate");
  AdjArgs a{batch, gH, gQ, gE, gd, grh, gke, gr};
  std::string err;
  int rc = launch_adjoint(plan->dn, plan->dw, a, plan->groups, stream, &err);
  if (rc != WDS_OK) return fail(rc, err);
  return WDS_OK;
}

extern "C" int wds_adjoint_pumps(WdsPlan* plan, int32_t batch, const double* gH,
                                 const double* gQ, const double* gE, double* gd, double* grh,
                                 double* gke, double* gr, double* gspeed, double* gh0,
                                 double* grp, void* stream) {
  using namespace wds;
  if (!plan || batch <= 0 || !gH || !gQ || !gE || !gd || !grh || !gke || !gr || !gspeed ||
      !gh0 || !grp)
    return fail(WDS_E_ARG, "wds_adjoint_pumps: bad argument");
  if (!plan->have_state || batch != plan->state_batch)
    return fail(WDS_E_STATE,
                "wds_adjoint_pumps: no implicit forward of this batch size to differentiate");
  AdjArgs a{batch, gH, gQ, gE, gd, grh, gke, gr};
  a.gsp = gspeed;
  a.gh0 = gh0;
  a.grp = grp;
  std::string err;
  int rc = launch_adjoint(plan->dn, plan->dw, a, plan->groups, stream, &err);
  if (rc != WDS_OK) return fail(rc, err);
  return WDS_OK;
}

extern "C" int wds_unrolled_adjoint(WdsPlan* plan, int32_t batch, int32_t K,
                                    const double* record, const double* demand,
                                    const double* fixed_head, const double* ke,
                                    int64_t ke_stride, const double* r, int64_t r_stride,
                                    const double* gH, const double* gQ, const double* gE,
                                    double* gd, double* grh, double* gke, double* gr,
                                    double* scratch, const int8_t* status0, void* stream) {
  using namespace wds;
  if (!plan || batch <= 0 || K <= 0 || !record || !demand || !fixed_head || !ke || !r || !gH ||
      !gQ || !gE || !gd || !grh || !gke || !gr || !scratch)
    return fail(WDS_E_ARG, "wds_unrolled_adjoint: bad argument");
  if (batch > plan->max_batch)
    return fail(WDS_E_ARG, "wds_unrolled_adjoint: batch exceeds the plan's max_batch");
  if (plan->dn.npcv > 0 || plan->dn.nfcv > 0)
    return fail(WDS_E_UNSUPPORTED,
                "wds_unrolled_adjoint: control valves (PRV/PSV/FCV) are not on the unrolled route");
  if ((ke_stride != 0 && ke_stride != plan->dn.N) || (r_stride != 0 && r_stride != plan->dn.L))
    return fail(WDS_E_ARG, "wds_unrolled_adjoint: ke_stride must be 0 or N, r_stride 0 or L");
  UnrollArgs u{};
  u.B = batch; u.K = K; u.rec = record; u.d = demand; u.rh = fixed_head; u.ke = ke;
  u.ke_stride = ke_stride; u.r = r; u.r_stride = r_stride; u.gH = gH; u.gQ = gQ; u.gE = gE;
  u.gd = gd; u.grh = grh; u.gke = gke; u.gr = gr; u.scr = scratch; u.s0 = status0;
  std::string err;
  const int rc = launch_unrolled(plan->dn, plan->dw, u, plan->groups, stream, &err);
  plan->have_state = false;  // the reverse pass reuses the plan's factor workspace
  ++plan->gen;
  if (rc != WDS_OK) return fail(rc, err);
  return WDS_OK;
}

extern "C" int wds_free(WdsPlan* plan) {
  if (!plan) return WDS_OK;
  if (plan->dtab) cudaFree(plan->dtab);
  if (plan->dwork) cudaFree(plan->dwork);
  delete plan;
  return WDS_OK;
}

// ---------------------------------------------------------------------------
// Forward without allocation.
//
// Some callers cannot call cudaMalloc when they solve: a pressure-management
// control loop that allocates everything at start-up because an allocation
// can stall it for milliseconds, or a host process whose device memory is
// owned by another allocator (a simulator or framework that hands this
// library only the buffers it asked for).  For them, wds_forward_noalloc runs
// the same forward kernel as wds_forward, but its per-scenario workspace (the
// polish's heads and Woodbury columns, the terminal factor and coefficients,
// the link flows) lives in the fixed array below instead of the plan's
// workspace, with the layout of work_layout.  The array is
// WDS_NOALLOC_SCRATCH_BYTES (64 MiB) and every GPU that loads this library
// holds it until the process exits.
//
// The kernel writes every word of the workspace it reads later in the same
// call, so nothing needs clearing between calls; the array keeps the last
// call's contents.  All calls share the one array: calls whose kernels
// overlap on the GPU (different streams, or different host threads) race on
// it and must be serialised by the caller.  A call does not prepare
// wds_adjoint; the plan's own state is left as it was.
static __device__ __align__(256) unsigned char g_noalloc_scratch[WDS_NOALLOC_SCRATCH_BYTES];

namespace {
// Device address of g_noalloc_scratch on the current device.  In host code
// the symbol is only a stand-in, not a device address, so it is looked up on
// every call (cheap, and it allocates nothing): a cached address could
// outlive the device context it came from (cudaDeviceReset).  The first
// lookup on a device loads this library's device code there, which creates
// the array.
int scratch_address(void** out) {
  void* p = nullptr;
  const cudaError_t ce = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (ce != cudaSuccess || !p)
    return fail(WDS_E_CUDA, std::string("wds_forward_noalloc: cudaGetSymbolAddress: ") +
                                cudaGetErrorString(ce));
  *out = p;
  return WDS_OK;
}
}  // namespace

extern "C" int wds_forward_noalloc(const WdsPlan* plan, int32_t batch, const WdsForwardOpts* o,
                                   const double* demand, const double* fixed_head,
                                   const double* ke, const double* r, double* head, double* flow,
                                   double* emitter, int8_t* status, int32_t* iters,
                                   double* relerr, int32_t* info, void* stream) {
  using namespace wds;
  if (!plan || !o || batch <= 0) return fail(WDS_E_ARG, "wds_forward_noalloc: bad argument");
  if (!demand || !fixed_head || !ke || !r || !head || !flow || !emitter || !status || !iters ||
      !relerr || !info)
    return fail(WDS_E_ARG, "wds_forward_noalloc: null pointer");
  if (o->max_iter <= 0 || !(o->accuracy > 0.0) || o->refine < 0)
    return fail(WDS_E_ARG, "wds_forward_noalloc: bad options");
  const DevNet& d = plan->dn;
  // the plan's workspace layout, for `batch` scenarios, inside the fixed array
  const WorkOff wo = work_layout(d, plan->dw.nscr, (size_t)batch, state_smem_bytes(d));
  if (wo.bytes > (size_t)WDS_NOALLOC_SCRATCH_BYTES) {
    const size_t per = wo.bytes / (size_t)batch;
    return fail(WDS_E_ARG, "wds_forward_noalloc: batch " + std::to_string(batch) + " needs " +
                               std::to_string(wo.bytes) + " bytes of scratch, the fixed array holds " +
                               std::to_string((size_t)WDS_NOALLOC_SCRATCH_BYTES) +
                               " (at most " + std::to_string(WDS_NOALLOC_SCRATCH_BYTES / per) +
                               " scenarios of this network)");
  }
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc != WDS_OK) return rc;
  const DevWork w = work_at((unsigned char*)base, wo, d, plan->dw.nscr);
  FwdArgs a{};
  a.B = batch; a.hacc = o->accuracy; a.max_iter = o->max_iter; a.sm = o->status_machine ? 1 : 0;
  a.refine = o->refine; a.polish = o->polish_steps; a.ke_stride = o->ke_stride;
  a.r_stride = o->r_stride; a.d = demand; a.rh = fixed_head; a.ke = ke; a.r = r;
  a.q0 = o->q0; a.e0 = o->e0;
  rc = set_pump_opts(a, o, d.L, "wds_forward_noalloc");
  if (rc != WDS_OK) return rc;
  a.head = head; a.flow = flow; a.emit = emitter; a.status = status; a.iters = iters;
  a.relerr = relerr; a.info = info;
  std::string err;
  rc = launch_forward(d, w, a, plan->groups, stream, &err);
  if (rc != WDS_OK) return fail(rc, err);
  return WDS_OK;
}
