// Fused batched GGA forward and reduced implicit adjoint for sm_100a.
//
// One CTA owns one scenario for the whole call: its link flows, link
// coefficients, the factor of the node matrix and the node vectors live in
// shared memory from the first Newton iteration to the terminal factorisation,
// so there is no host round trip and no HBM traffic inside the loop.
//
// Per GGA iteration (dgga/solver.py:2922-3179):
//   link pass    P, Y from the headloss formulas (one thread per link)
//   node pass    gather assembly of A (diagonal, pairs) and F in the
//                reference's scatter order; PRV valve coefficients after the
//                node coefficients (serial over the few PRVs)
//   factor       left-looking LDL^T, one barrier per elimination-tree level
//   solve        level-scheduled forward/backward substitution + refinement
//                against the matrix-free operator A x
//   update       dq = Y - P dh, emitter update, relerr reduction, status
//                machine (valve status every iteration, link status on the
//                converged / periodic branches, per-scenario nextcheck)
// Implicit mode then runs the reduced Newton polish with Woodbury row
// replacement for ACTIVE PRVs (dgga/autodiff.py:965-1104) and stores the
// terminal factor and coefficients for the adjoint kernel.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "wds_internal.h"

namespace wds {
namespace {

constexpr double kINF = __builtin_huge_val();

struct Sh {
  double *q, *P, *Y, *W, *V0, *V1, *V2, *e, *emh, *hf, *xf, *red, *small;
  int8_t* S;
};

__device__ __forceinline__ double head_of(int c, const double* x, const double* hf) {
  return c >= 0 ? x[c] : hf[-c - 1];
}
__device__ __forceinline__ double junc_of(int c, const double* x) { return c >= 0 ? x[c] : 0.0; }

// ---------------------------------------------------------------- reductions
template <int NT>
__device__ void block_sum(double* v, int m, double* red) {
  for (int i = 0; i < m; ++i)
    for (int o = 16; o; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0)
    for (int i = 0; i < m; ++i) red[w * 4 + i] = v[i];
  __syncthreads();
  for (int i = 0; i < m; ++i) {
    double s = 0.0;
    for (int ww = 0; ww < NT / 32; ++ww) s += red[ww * 4 + i];
    v[i] = s;
  }
}

// ---------------------------------------------------------------- formulas
// emitterheadloss (dgga/solver.py:2368-2377)
__device__ __forceinline__ void emitter_hl(const DevNet& n, double e, double ke, double& hl,
                                           double& hg) {
  const double kea = fmax(ke, kCSMALL);
  hg = n.qexp * kea * pow(fmax(fabs(e), 1e-30), n.qexp - 1.0);
  const bool lin = hg < n.rqtol;
  if (lin) hg = n.rqtol;
  hl = lin ? hg * e : hg * e / n.qexp;
}

// valvecoeff open branch (dgga/solver.py:2203-2219, :834-848)
__device__ __forceinline__ void valve_open(const DevNet& n, double q, double km, double& P,
                                           double& Y) {
  double hg = 2.0 * km * fabs(q);
  const bool lin = hg < n.rqtol;
  if (lin) hg = n.rqtol;
  const double hl = lin ? q * hg : q * hg / 2.0;
  if (km > 0.0) {
    P = 1.0 / hg;
    Y = hl / hg;
  } else {
    P = 1.0 / kCSMALL;
    Y = q;
  }
}

// pipecoeff, Hazen-Williams / Chezy-Manning (dgga/solver.py:2176-2201)
__device__ __forceinline__ void pipe_coef(const DevNet& n, double q, double r, double km,
                                          double& P, double& Y) {
  const double sgn = q < 0.0 ? -1.0 : 1.0;
  const double qa = q * sgn;
  double hg = n.hexp * r * pow(fmax(qa, 1e-30), n.hexp - 1.0);
  const bool lin = hg < n.rqtol;
  if (lin) hg = n.rqtol;
  double hl = lin ? hg * qa : hg * qa / n.hexp;
  if (km > 0.0) {
    hl = hl + km * qa * qa;
    hg = hg + 2.0 * km * qa;
  }
  hl = hl * sgn;
  P = 1.0 / hg;
  Y = hl / hg;
}

// pumpcoeff for every curve kind (dgga/solver.py:2221-2326)
__device__ void pump_coef(const DevNet& n, int k, double q, double& P, double& Y) {
  const int t = n.ptype[k];
  if (t == 3) {  // NOCURVE: an open valve
    P = 1.0 / kCSMALL;
    Y = q;
    return;
  }
  const double sgn = q < 0.0 ? -1.0 : 1.0;
  const double qa = q * sgn;
  const double spc = fmax(n.pspeed[k], 1e-12);
  double hg, hl;
  if (t == 2) {  // CUSTOM: piecewise-linear curve segment
    const int c0 = n.cptr[k], np = n.cptr[k + 1] - c0;
    const double* X = n.cx + c0;
    const double* Yc = n.cy + c0;
    const double qq = (fabs(q) / spc) * n.ucf_flow;
    int idx = 0;
    while (idx < np && X[idx] < qq) ++idx;
    const int k2 = min(max(idx, 1), np - 1), k1 = k2 - 1;
    double rc = (Yc[k2] - Yc[k1]) / (X[k2] - X[k1]);
    double h0c = Yc[k1] - rc * X[k1];
    h0c = h0c / n.ucf_head;
    rc = rc * n.ucf_flow / n.ucf_head;
    hg = (-rc) * spc;
    hl = (-h0c) * (spc * spc) + hg * q;
  } else {
    const double pn = n.pn[k];
    const double h0e = spc * spc * n.ph0[k];
    const double re = n.pr[k] * pow(spc, 2.0 - pn);
    if (t == 0) {  // CONST_HP
      const double qac = fmax(qa, 1e-30);
      const double raw = -re / qac / qac;
      const bool big = raw > kCBIG, sml = raw < n.rqtol;
      hg = big ? kCBIG : (sml ? n.rqtol : raw);
      hl = (big || sml) ? -hg * q : re / (sgn * qac);
    } else if (pn == 1.0) {  // linear power function
      hg = re;
      hl = h0e + re * q;
    } else {  // power function; pow(0, n-1) taken exactly
      const double nm1 = pn - 1.0;
      double pw;
      if (qa == 0.0)
        pw = nm1 > 0.0 ? 0.0 : ((nm1 < 0.0 && t == 1) ? kINF : 1.0);
      else
        pw = pow(qa, nm1);
      const double raw = pn * re * pw;
      const bool sml = raw < n.rqtol;
      hg = sml ? n.rqtol : raw;
      hl = sml ? h0e + hg * q : h0e + hg * q / fmax(pn, 1e-30);
    }
  }
  P = 1.0 / hg;
  Y = hl / hg;
}

// PRV valve coefficients of one status-machine PRV (dgga/solver.py:862-903):
// returns pna (the non-ACTIVE P, zero when ACTIVE) and yna.
__device__ __forceinline__ void prv_open(const DevNet& n, int i, double qk, int sk, double& pna,
                                         double& yna) {
  const bool act = sk == WDS_ACTIVE, cl = sk <= WDS_CLOSED;
  const double km = n.pcv_km[i];
  double po, yo;
  if (km > 0.0) {
    double hg = 2.0 * km * fabs(qk);
    const bool lin = hg < n.rqtol;
    if (lin) hg = n.rqtol;
    const double hl = lin ? qk * hg : qk * hg / 2.0;
    po = 1.0 / hg;
    yo = hl / hg;
  } else {
    po = 1.0 / kCSMALL;
    yo = qk;
  }
  pna = (cl ? 1.0 / kCBIG : po) * (act ? 0.0 : 1.0);
  yna = cl ? qk : yo;
}

// Link coefficients of the headloss stage (dgga/solver.py:2923-2956).
// `adj` selects the adjoint/polish variant in which a status-machine PRV
// takes its valve coefficients directly (autodiff.py:838-847).
__device__ __forceinline__ void link_coef(const DevNet& n, int k, double q, int s, double r,
                                          bool adj, double& P, double& Y) {
  const int kd = n.kind[k];
  if (kd == WDS_KIND_PRV) {
    if (!adj) {
      P = 0.0;
      Y = 0.0;
    } else {
      double pna, yna;
      prv_open(n, n.link_pcv[k], q, s, pna, yna);
      P = pna;
      Y = (s == WDS_ACTIVE) ? q + 0.0 : yna;
    }
    return;
  }
  if (s <= WDS_CLOSED || (n.flags[k] & WDS_F_ZERO_SPEED)) {
    P = 1.0 / kCBIG;
    Y = q;
    return;
  }
  if (kd <= WDS_KIND_CVPIPE)
    pipe_coef(n, q, r, n.km[k], P, Y);
  else if (kd == WDS_KIND_TCV)
    valve_open(n, q, n.km_tcv[k], P, Y);
  else if (kd == WDS_KIND_PRV_FIXED)
    valve_open(n, q, n.km[k], P, Y);
  else
    pump_coef(n, k, q, P, Y);
}

// ---------------------------------------------------------------- linear algebra
// Matrix-free (A x)_p of the node matrix: links with conductance P, emitter
// diagonal emh, CBIG on the downstream node of ACTIVE PRVs
// (dgga/autodiff.py:878-895; the same operator the forward assembles).
__device__ __forceinline__ double amul_node(const DevNet& n, int p, const double* P,
                                            const double* x, const double* emh,
                                            const int8_t* S) {
  double acc = 0.0;
  const int a = n.inc_ptr[p], m = n.inc_split[p], z = n.inc_ptr[p + 1];
  for (int e = a; e < m; ++e) {
    const int k = n.inc[e];
    acc += P[k] * (junc_of(n.e1[k], x) - junc_of(n.e2[k], x));
  }
  for (int e = m; e < z; ++e) {
    const int k = n.inc[e];
    acc += -(P[k] * (junc_of(n.e1[k], x) - junc_of(n.e2[k], x)));
  }
  acc = acc + emh[p] * x[p];
  for (int c = n.cb_ptr[p]; c < n.cb_ptr[p + 1]; ++c) {
    const int i = n.cb_idx[c];
    const double act = S[n.pcv_link[i]] == WDS_ACTIVE ? 1.0 : 0.0;
    acc += x[p] * act * kCBIG;
  }
  return acc;
}

// Left-looking LDL^T by elimination-tree level.  W holds A on entry (pattern
// of L, fill zero) and on exit the unscaled columns L_ij D_j with 1/D_j in the
// diagonal slot.  Returns true when every pivot was positive and finite.
template <int NT>
__device__ bool ldl_factor(const DevNet& n, double* W) {
  bool bad = false;
  for (int lv = 0; lv < n.nlev; ++lv) {
    const int t0 = n.ftask_ptr[lv], t1 = n.ftask_ptr[lv + 1];
    for (int t = t0 + threadIdx.x; t < t1; t += NT) {
      const int4 tk = n.ftask[t];
      double w = W[tk.x];
      for (int pr = tk.y; pr < tk.z; ++pr) {
        const int* f = n.fpair + 3 * pr;
        w -= W[f[0]] * W[f[1]] * W[f[2]];
      }
      if (tk.w) {
        if (!(w > 0.0) || !isfinite(w)) bad = true;
        W[tk.x] = 1.0 / w;
      } else {
        W[tk.x] = w;
      }
    }
    __syncthreads();
  }
  return !__syncthreads_or(bad);
}

// In-place solve of (L D L^T) v = b, level-scheduled.
template <int NT>
__device__ void ldl_solve(const DevNet& n, const double* W, double* v) {
  for (int lv = 0; lv < n.nlev; ++lv) {
    for (int t = n.levptr[lv] + threadIdx.x; t < n.levptr[lv + 1]; t += NT) {
      const int j = n.levcol[t];
      double acc = v[j];
      for (int e = n.rptr[j]; e < n.rptr[j + 1]; ++e) acc -= W[n.rslot[e]] * v[n.rcol[e]];
      v[j] = acc * W[n.colptr[j]];
    }
    __syncthreads();
  }
  for (int lv = n.nlev - 1; lv >= 0; --lv) {
    for (int t = n.levptr[lv] + threadIdx.x; t < n.levptr[lv + 1]; t += NT) {
      const int j = n.levcol[t];
      const int c0 = n.colptr[j];
      double s = 0.0;
      for (int e = c0 + 1; e < n.colptr[j + 1]; ++e) s += W[e] * v[n.rowidx[e]];
      v[j] = v[j] - W[c0] * s;
    }
    __syncthreads();
  }
}

// x = A^{-1} rhs with `refine` refinement steps against the matrix-free A.
template <int NT>
__device__ void solve_refined(const DevNet& n, const double* W, const double* P,
                              const double* emh, const int8_t* S, const double* rhs, double* x,
                              double* t, int refine) {
  for (int p = threadIdx.x; p < n.Nj; p += NT) x[p] = rhs[p];
  __syncthreads();
  ldl_solve<NT>(n, W, x);
  for (int it = 0; it < refine; ++it) {
    for (int p = threadIdx.x; p < n.Nj; p += NT)
      t[p] = rhs[p] - amul_node(n, p, P, x, emh, S);
    __syncthreads();
    ldl_solve<NT>(n, W, t);
    for (int p = threadIdx.x; p < n.Nj; p += NT) x[p] = x[p] + t[p];
    __syncthreads();
  }
}

// Small dense solve (Gaussian elimination, partial pivoting), one thread.
__device__ void dense_solve(double* C, double* y, int m) {
  for (int c = 0; c < m; ++c) {
    int piv = c;
    for (int r = c + 1; r < m; ++r)
      if (fabs(C[r * m + c]) > fabs(C[piv * m + c])) piv = r;
    if (piv != c) {
      for (int k = 0; k < m; ++k) {
        double tmp = C[c * m + k];
        C[c * m + k] = C[piv * m + k];
        C[piv * m + k] = tmp;
      }
      double tmp = y[c];
      y[c] = y[piv];
      y[piv] = tmp;
    }
    for (int r = c + 1; r < m; ++r) {
      const double f = C[r * m + c] / C[c * m + c];
      for (int k = c; k < m; ++k) C[r * m + k] -= f * C[c * m + k];
      y[r] -= f * y[c];
    }
  }
  for (int c = m - 1; c >= 0; --c) {
    double s = y[c];
    for (int k = c + 1; k < m; ++k) s -= C[c * m + k] * y[k];
    y[c] = s / C[c * m + c];
  }
}

// ---------------------------------------------------------------- assembly
// GGA assembly (linkcoeffs -> emittercoeffs -> nodecoeffs, solver.py:2958-3007)
// into W (pattern of L) and F; Xflow saved for PRV downstream nodes.
template <int NT>
__device__ void assemble_gga(const DevNet& n, const Sh& s, const double* kerow,
                             const double* drow) {
  for (int p = threadIdx.x; p < n.Nj; p += NT) {
    const int a = n.inc_ptr[p], m = n.inc_split[p], z = n.inc_ptr[p + 1];
    double dg = 0.0, xf = 0.0, F = 0.0;
    for (int e = a; e < m; ++e) {
      const int k = n.inc[e];
      if (n.kind[k] == WDS_KIND_PRV) continue;
      dg += s.P[k];
      xf += -s.q[k];
      F += s.Y[k];
    }
    for (int e = m; e < z; ++e) {
      const int k = n.inc[e];
      if (n.kind[k] == WDS_KIND_PRV) continue;
      dg += s.P[k];
      xf += s.q[k];
      F += -s.Y[k];
    }
    for (int e = m; e < z; ++e) {  // n1 end fixed: F[Row[n2]] += P*H[n1]
      const int k = n.inc[e];
      if (n.kind[k] == WDS_KIND_PRV || n.e1[k] >= 0) continue;
      F += s.P[k] * s.hf[-n.e1[k] - 1];
    }
    for (int e = a; e < m; ++e) {  // n2 end fixed: F[Row[n1]] += P*H[n2]
      const int k = n.inc[e];
      if (n.kind[k] == WDS_KIND_PRV || n.e2[k] >= 0) continue;
      F += s.P[k] * s.hf[-n.e2[k] - 1];
    }
    const double ke = kerow[n.jnode[p]];
    double emh = 0.0;
    if (ke > 0.0) {
      double hl, hg;
      emitter_hl(n, s.e[p], ke, hl, hg);
      emh = 1.0 / hg;
      dg = dg + emh;
      F = F + (hl + n.el[p]) / hg;
      xf = xf - s.e[p];
    }
    s.emh[p] = emh;
    xf = xf - drow[n.jnode[p]];
    F = F + xf;
    s.W[n.colptr[p]] = dg;
    s.V0[p] = F;
    if (n.node_xf[p] >= 0) s.xf[n.node_xf[p]] = xf;
  }
  for (int t = threadIdx.x; t < n.npairs; t += NT) {
    double v = 0.0;
    for (int e = n.pair_ptr[t]; e < n.pair_ptr[t + 1]; ++e) {
      const int k = n.pair_link[e];
      if (n.kind[k] == WDS_KIND_PRV) continue;
      v += -s.P[k];
    }
    s.W[n.pair_slot[t]] = v;
  }
  for (int t = threadIdx.x; t < n.nfill; t += NT) s.W[n.fill_slot[t]] = 0.0;
  __syncthreads();
  if (threadIdx.x == 0) {  // valvecoeffs after nodecoeffs, in valve order
    for (int i = 0; i < n.npcv; ++i) {
      const int k = n.pcv_link[i];
      const double qk = s.q[k];
      const int sk = s.S[k];
      const bool act = sk == WDS_ACTIVE;
      double pna, yna;
      prv_open(n, i, qk, sk, pna, yna);
      const double mna = act ? 0.0 : 1.0, mact = act ? 1.0 : 0.0;
      const double xf2 = s.xf[n.pcv_xf[i]];
      const double dy = (yna - qk) * mna;
      const double f1 = dy + ((act && xf2 < 0.0) ? xf2 : 0.0);
      const double f2 = -dy + n.pcv_hset[i] * kCBIG * mact;
      const int j1 = n.pcv_j1[i], j2 = n.pcv_j2[i];
      s.W[n.pcv_off[i]] += -pna;
      s.W[n.colptr[j1]] += pna;
      s.W[n.colptr[j2]] += pna;
      s.W[n.colptr[j2]] += kCBIG * mact;
      s.V0[j1] += f1;
      s.V0[j2] += f2;
      s.P[k] = pna;
      s.Y[k] = act ? qk + xf2 : yna;
    }
  }
  __syncthreads();
}

// Reduced-matrix assembly at the current state (dgga/autodiff.py:928-962):
// every link with its P, + emh diagonal, + CBIG on ACTIVE PRV downstream nodes.
template <int NT>
__device__ void assemble_reduced(const DevNet& n, const Sh& s) {
  for (int p = threadIdx.x; p < n.Nj; p += NT) {
    double dg = 0.0;
    for (int e = n.inc_ptr[p]; e < n.inc_ptr[p + 1]; ++e) dg += s.P[n.inc[e]];
    dg = dg + s.emh[p];
    for (int c = n.cb_ptr[p]; c < n.cb_ptr[p + 1]; ++c) {
      const int i = n.cb_idx[c];
      dg += kCBIG * (s.S[n.pcv_link[i]] == WDS_ACTIVE ? 1.0 : 0.0);
    }
    s.W[n.colptr[p]] = dg;
  }
  for (int t = threadIdx.x; t < n.npairs; t += NT) {
    double v = 0.0;
    for (int e = n.pair_ptr[t]; e < n.pair_ptr[t + 1]; ++e) v += -s.P[n.pair_link[e]];
    s.W[n.pair_slot[t]] = v;
  }
  for (int t = threadIdx.x; t < n.nfill; t += NT) s.W[n.fill_slot[t]] = 0.0;
  __syncthreads();
}

// Coefficients at the current state for polish / terminal (autodiff.py:786-875):
// P, Y per link; emh per junction.
template <int NT>
__device__ void adj_coeffs(const DevNet& n, const Sh& s, const double* rrow,
                           const double* kerow) {
  for (int k = threadIdx.x; k < n.L; k += NT) {
    double P, Y;
    link_coef(n, k, s.q[k], s.S[k], rrow[k], true, P, Y);
    s.P[k] = P;
    s.Y[k] = Y;
  }
  for (int p = threadIdx.x; p < n.Nj; p += NT) {
    const double ke = kerow[n.jnode[p]];
    double emh = 0.0;
    if (ke > 0.0) {
      double hl, hg;
      emitter_hl(n, s.e[p], ke, hl, hg);
      emh = 1.0 / hg;
    }
    s.emh[p] = emh;
  }
  __syncthreads();
}

// Woodbury data for ACTIVE-PRV rows.
struct Wood {
  double* cols;  // [m][Nj] columns A^{-1} e_u
  double* C;     // [m*m] in shared memory (small)
  int m;
};

// Primal reduced Newton solve with ACTIVE-PRV Dirichlet / merged rows
// (dgga/autodiff.py:965-1029).  rhs: V0 (kept), result in dH.
template <int NT>
__device__ void primal_solve(const DevNet& n, const Sh& s, double* rp, double* dH,
                             double* res, double* sx, double* cols, const double* rprv,
                             bool any_act, int refine) {
  const double* rhs = s.V0;
  double* t = s.V2;
  if (!any_act) {
    solve_refined<NT>(n, s.W, s.P, s.emh, s.S, rhs, dH, t, refine);
    return;
  }
  const int p = n.npcv, m = 2 * p;
  double* C = s.small;            // m*m
  double* y = s.small + m * m;    // m
  double* actf = y + m;           // p
  if (threadIdx.x == 0)
    for (int i = 0; i < p; ++i) actf[i] = s.S[n.pcv_link[i]] == WDS_ACTIVE ? 1.0 : 0.0;
  for (int q = threadIdx.x; q < n.Nj; q += NT) rp[q] = rhs[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    // rp[j1] += rhs[j2] (ACTIVE), then rp[j2] = -r_prv
    for (int i = 0; i < p; ++i)
      if (actf[i] != 0.0) rp[n.pcv_j1[i]] += rhs[n.pcv_j2[i]];
    for (int i = 0; i < p; ++i)
      if (actf[i] != 0.0) rp[n.pcv_j2[i]] = -rprv[i];
  }
  __syncthreads();
  solve_refined<NT>(n, s.W, s.P, s.emh, s.S, rp, dH, t, refine);
  for (int c = 0; c < m; ++c) {
    const int u = c < p ? n.pcv_j2[c] : n.pcv_j1[c - p];
    for (int q = threadIdx.x; q < n.Nj; q += NT) res[q] = q == u ? 1.0 : 0.0;
    __syncthreads();
    solve_refined<NT>(n, s.W, s.P, s.emh, s.S, res, cols + (size_t)c * n.Nj, t, refine);
  }
  if (threadIdx.x == 0) {
    // C = [R2 ; I2 - CBIG R2], rows of inactive valves -> identity
    for (int a = 0; a < p; ++a)
      for (int c = 0; c < m; ++c) {
        const double r2 = cols[(size_t)c * n.Nj + n.pcv_j2[a]];
        const double i2 = (c == a || c == a + p) ? 1.0 : 0.0;
        C[a * m + c] = actf[a] != 0.0 ? r2 : (c == a ? 1.0 : 0.0);
        C[(a + p) * m + c] = actf[a] != 0.0 ? i2 - kCBIG * r2 : (c == a + p ? 1.0 : 0.0);
      }
  }
  __syncthreads();
  // x <- x - S y,  y = C^{-1} [ (x[j2]-rr[j2]) act ; (rr[j2] - CBIG x[j2]) act ]
  auto wood = [&](double* x, const double* rr) {
    if (threadIdx.x == 0) {
      double Cc[64];
      for (int i = 0; i < m * m; ++i) Cc[i] = C[i];
      for (int a = 0; a < p; ++a) {
        const int j2 = n.pcv_j2[a];
        y[a] = (x[j2] - rr[j2]) * actf[a];
        y[a + p] = (rr[j2] - kCBIG * x[j2]) * actf[a];
      }
      dense_solve(Cc, y, m);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n.Nj; q += NT) {
      double acc = 0.0;
      for (int c = 0; c < m; ++c) acc += cols[(size_t)c * n.Nj + q] * y[c];
      x[q] = x[q] - acc;
    }
    __syncthreads();
  };
  wood(dH, rp);
  double* row1 = actf + p;  // p
  for (int it = 0; it < 2; ++it) {
    for (int q = threadIdx.x; q < n.Nj; q += NT) res[q] = amul_node(n, q, s.P, dH, s.emh, s.S);
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < p; ++i)
        row1[i] = res[n.pcv_j1[i]] + res[n.pcv_j2[i]] - kCBIG * dH[n.pcv_j2[i]];
    __syncthreads();
    for (int q = threadIdx.x; q < n.Nj; q += NT) res[q] = rp[q] - res[q];
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int i = 0; i < p; ++i)
        if (actf[i] != 0.0) res[n.pcv_j1[i]] = rp[n.pcv_j1[i]] - row1[i];
      for (int i = 0; i < p; ++i)
        if (actf[i] != 0.0) res[n.pcv_j2[i]] = rp[n.pcv_j2[i]] - dH[n.pcv_j2[i]];
    }
    __syncthreads();
    solve_refined<NT>(n, s.W, s.P, s.emh, s.S, res, sx, t, refine);
    wood(sx, res);
    for (int q = threadIdx.x; q < n.Nj; q += NT) dH[q] = dH[q] + sx[q];
    __syncthreads();
  }
}

__device__ __forceinline__ size_t al16(size_t x) { return (x + 15) / 16 * 16; }

__device__ Sh carve(const DevNet& n, unsigned char* base) {
  Sh s;
  size_t o = 0;
  auto take = [&](size_t bytes) { unsigned char* p = base + o; o = al16(o + bytes); return p; };
  s.q = (double*)take(8ull * n.L);
  s.P = (double*)take(8ull * n.L);
  s.Y = (double*)take(8ull * n.L);
  s.W = (double*)take(8ull * n.nnzL);
  s.V0 = (double*)take(8ull * n.Nj);
  s.V1 = (double*)take(8ull * n.Nj);
  s.V2 = (double*)take(8ull * n.Nj);
  s.e = (double*)take(8ull * n.Nj);
  s.emh = (double*)take(8ull * n.Nj);
  s.hf = (double*)take(8ull * (n.Nf > 0 ? n.Nf : 1));
  s.xf = (double*)take(8ull * (n.nxf > 0 ? n.nxf : 1));
  s.red = (double*)take(8ull * 4 * 32);
  s.small = (double*)take(8ull * (4 * n.npcv * n.npcv + 5 * n.npcv + 8));
  s.S = (int8_t*)take(n.L);
  return s;
}

// ---------------------------------------------------------------- forward kernel
template <int NT>
__global__ void __launch_bounds__(NT) k_forward(DevNet n, DevWork w, FwdArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int b = blockIdx.x;
  Sh s = carve(n, smem_raw);
  const double* rrow = a.r + (long long)b * a.r_stride;
  const double* kerow = a.ke + (long long)b * a.ke_stride;
  const double* drow = a.d + (long long)b * n.N;
  const double* rhrow = a.rh + (long long)b * n.N;
  for (int f = threadIdx.x; f < n.Nf; f += NT) s.hf[f] = rhrow[n.fnode[f]];
  for (int k = threadIdx.x; k < n.L; k += NT) {
    s.q[k] = n.q_init[k];
    s.S[k] = n.status0[k];
  }
  for (int p = threadIdx.x; p < n.Nj; p += NT) s.e[p] = kerow[n.jnode[p]] > 0.0 ? 1.0 : 0.0;
  __syncthreads();
  const bool sm = a.sm != 0;
  const int maxtrials = sm ? a.max_iter + (n.extra_iter > 0 ? n.extra_iter : 0) : a.max_iter;
  int nextcheck = n.checkfreq;
  int iters = maxtrials + 1, info = WDS_INFO_UNCONVERGED;
  double relerr = 0.0;
  for (int it = 1; it <= maxtrials; ++it) {
    // ---- headloss coefficients
    for (int k = threadIdx.x; k < n.L; k += NT) {
      double P, Y;
      link_coef(n, k, s.q[k], s.S[k], rrow[k], false, P, Y);
      s.P[k] = P;
      s.Y[k] = Y;
    }
    __syncthreads();
    assemble_gga<NT>(n, s, kerow, drow);
    if (!ldl_factor<NT>(n, s.W)) {
      info = WDS_INFO_NOT_PD;
      iters = it;
      break;
    }
    solve_refined<NT>(n, s.W, s.P, s.emh, s.S, s.V0, s.V1, s.V2, a.refine);
    // ---- newflows (hydsolver.c:358-514 as restated in solver.py:3092-3110)
    double sums[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = threadIdx.x; k < n.L; k += NT) {
      const double dh = head_of(n.e1[k], s.V1, s.hf) - head_of(n.e2[k], s.V1, s.hf);
      double dq = s.Y[k] - s.P[k] * dh;
      if ((n.flags[k] & WDS_F_CHP) && dq > s.q[k]) dq = s.q[k] / 2.0;
      const double qn = s.q[k] - dq;
      s.q[k] = qn;
      sums[0] += fabs(dq);
      sums[1] += fabs(qn);
    }
    for (int p = threadIdx.x; p < n.Nj; p += NT) {
      const double ke = kerow[n.jnode[p]];
      if (ke > 0.0) {
        double hl, hg;
        emitter_hl(n, s.e[p], ke, hl, hg);
        const double dqe = (hl - (s.V1[p] - n.el[p])) / hg;
        const double en = s.e[p] - dqe;
        s.e[p] = en;
        sums[2] += fabs(dqe);
        sums[3] += fabs(en);
      }
    }
    block_sum<NT>(sums, 4, s.red);
    const double dqsum = sums[0] + sums[2], qsum = sums[1] + sums[3];
    relerr = qsum > a.hacc ? dqsum / qsum : dqsum;
    if (!sm) {
      if (!(relerr > a.hacc)) {
        iters = it;
        info = 0;
        break;
      }
      continue;
    }
    // ---- batched status machine (hydsolve, solver.py:3126-3179)
    bool vchg = false;
    for (int i = threadIdx.x; i < n.npcv; i += NT) {
      const int k = n.pcv_link[i];
      const double h1 = head_of(n.e1[k], s.V1, s.hf), h2 = head_of(n.e2[k], s.V1, s.hf);
      const double qk = s.q[k], hs = n.pcv_hset[i], ht = n.htol;
      const int sk = s.S[k];
      const double hml = n.pcv_km[i] * (qk * qk);
      const bool neg = qk < -n.qtol;
      int ns = sk;
      if (sk == WDS_ACTIVE)
        ns = neg ? WDS_CLOSED : (h1 - hml < hs - ht ? WDS_OPEN : WDS_ACTIVE);
      else if (sk == WDS_OPEN)
        ns = neg ? WDS_CLOSED : (h2 >= hs + ht ? WDS_ACTIVE : WDS_OPEN);
      else if (sk == WDS_CLOSED)
        ns = (h1 >= hs + ht && h2 < hs - ht) ? WDS_ACTIVE
             : ((h1 < hs - ht && h1 > h2 + ht) ? WDS_OPEN : WDS_CLOSED);
      else if (sk == WDS_XPRESSURE)
        ns = neg ? WDS_CLOSED : sk;
      if (ns != sk) vchg = true;
      s.S[k] = (int8_t)ns;
    }
    vchg = __syncthreads_or(vchg);
    const bool conv = relerr <= a.hacc;
    const bool br_conv = conv && it <= a.max_iter;
    const bool br_per = !conv && it <= n.maxcheck && nextcheck == it;
    bool chg = false;
    if (br_conv || br_per) {
      for (int k = threadIdx.x; k < n.L; k += NT) {
        const int st0 = s.S[k];
        int st = (st0 == WDS_XHEAD || st0 == WDS_TEMPCLOSED) ? WDS_OPEN : st0;
        const double dh = head_of(n.e1[k], s.V1, s.hf) - head_of(n.e2[k], s.V1, s.hf);
        const double qk = s.q[k];
        if (n.kind[k] == WDS_KIND_CVPIPE) {  // cvstatus
          const bool rev = qk < -n.qtol;
          if (fabs(dh) > n.htol)
            st = (dh < -n.htol || rev) ? WDS_CLOSED : WDS_OPEN;
          else if (rev)
            st = WDS_CLOSED;
        }
        if ((n.flags[k] & WDS_F_PUMP_LIVE) && st >= WDS_OPEN)  // pumpstatus
          st = (-dh > n.phmax[k] + n.htol) ? WDS_XHEAD : WDS_OPEN;
        const int t = n.link_tl[k];
        if (t >= 0) {  // tankstatus
          const bool live = st > WDS_CLOSED;
          const double ht = s.hf[n.tl_tank[t]];
          const double dht = ht - head_of(n.tl_other[t], s.V1, s.hf);
          const double qq = qk * n.tl_qsign[t];
          const uint8_t fl = n.tl_flags[t];
          const bool full = (ht >= n.tl_hmax[t] - n.htol) && !(fl & WDS_TL_OVERFLOW);
          const bool empty = ht <= n.tl_hmin[t] + n.htol;
          const bool big = fabs(dht) > n.htol;
          const bool cbig = (dht < -n.htol) || (qq < -n.qtol);
          const bool cl_open = big ? cbig : (qq < -n.qtol);   // cvstatus from OPEN
          const bool cl_closed = big ? cbig : true;           // cvstatus from CLOSED
          const bool cut_f = (fl & WDS_TL_IS_PUMP) ? (fl & WDS_TL_PUMP_IN) != 0 : cl_open;
          const bool cut_e = (fl & WDS_TL_IS_PUMP) ? (fl & WDS_TL_PUMP_OUT) != 0 : !cl_closed;
          if (live && ((full && cut_f) || (empty && cut_e))) st = WDS_TEMPCLOSED;
        }
        if (st != st0) chg = true;
        s.S[k] = (int8_t)st;
      }
      chg = __syncthreads_or(chg);
    }
    const bool stat_change = br_conv && (chg || vchg);
    if (br_conv && stat_change) nextcheck = it + n.checkfreq;
    if (br_per) nextcheck += n.checkfreq;
    if (conv && (it > a.max_iter || !stat_change)) {
      iters = it;
      info = 0;
      break;
    }
  }
  __syncthreads();
  // junction heads of the GGA solution stay in V1
  double* Hs = w.scr + (size_t)b * w.nscr * n.Nj;  // global copy of heads for the polish
  if (a.polish >= 0 && info == 0) {
    for (int p = threadIdx.x; p < n.Nj; p += NT) Hs[p] = s.V1[p];
    __syncthreads();
    double* rp = Hs + n.Nj;
    double* res = rp + n.Nj;
    double* sx = res + n.Nj;
    double* cols = sx + n.Nj;
    // small buffer: C [4p^2], y [2p], actf [p], row1 [p], then r_prv [p]
    double* rprv = s.small + 4 * n.npcv * n.npcv + 4 * n.npcv;
    for (int step = 0; step <= a.polish; ++step) {
      adj_coeffs<NT>(n, s, rrow, kerow);
      assemble_reduced<NT>(n, s);
      if (!ldl_factor<NT>(n, s.W)) {
        info = WDS_INFO_NOT_PD;
        break;
      }
      if (step == a.polish) break;  // terminal factor: keep it
      // residuals (autodiff.py:1032-1050); r_l overwrites Y
      for (int k = threadIdx.x; k < n.L; k += NT) {
        const double hl = s.P[k] != 0.0 ? s.Y[k] / s.P[k] : 0.0;
        s.Y[k] = hl - (head_of(n.e1[k], Hs, s.hf) - head_of(n.e2[k], Hs, s.hf));
      }
      bool any_act = false;
      for (int i = threadIdx.x; i < n.npcv; i += NT) {
        const bool act = s.S[n.pcv_link[i]] == WDS_ACTIVE;
        rprv[i] = (Hs[n.pcv_j2[i]] - n.pcv_hset[i]) * (act ? 1.0 : 0.0);
        any_act |= act;
      }
      any_act = __syncthreads_or(any_act);
      for (int p = threadIdx.x; p < n.Nj; p += NT) {
        const int a0 = n.inc_ptr[p], m = n.inc_split[p], z = n.inc_ptr[p + 1];
        double mm = 0.0, bt = 0.0;
        for (int e = m; e < z; ++e) {
          const int k = n.inc[e];
          mm += s.q[k];
          bt += s.P[k] * s.Y[k];
        }
        for (int e = a0; e < m; ++e) {
          const int k = n.inc[e];
          mm += -s.q[k];
          bt += -(s.P[k] * s.Y[k]);
        }
        const double ke = kerow[n.jnode[p]];
        double re = 0.0;
        if (ke > 0.0) {
          double hl, hg;
          emitter_hl(n, s.e[p], ke, hl, hg);
          re = hl - (Hs[p] - n.el[p]);
          mm = mm - s.e[p];
        }
        mm = mm - drow[n.jnode[p]];
        s.V0[p] = (mm - bt) + s.emh[p] * re;
      }
      __syncthreads();
      primal_solve<NT>(n, s, rp, s.V1, res, sx, cols, rprv, any_act, a.refine);
      // dq, de, state update
      for (int k = threadIdx.x; k < n.L; k += NT) {
        const double b1 = junc_of(n.e1[k], s.V1), b2 = junc_of(n.e2[k], s.V1);
        double dq = -s.P[k] * (s.Y[k] + (b2 - b1));
        const int i = n.link_pcv[k];
        if (i >= 0 && s.S[k] == WDS_ACTIVE) {
          const int j2 = n.pcv_j2[i];
          const double ab2 = amul_node(n, j2, s.P, s.V1, s.emh, s.S) - kCBIG * s.V1[j2] * 1.0;
          dq = s.V0[j2] - ab2;
        }
        s.q[k] = s.q[k] + dq;
      }
      for (int p = threadIdx.x; p < n.Nj; p += NT) {
        const double ke = kerow[n.jnode[p]];
        if (ke > 0.0) {
          double hl, hg;
          emitter_hl(n, s.e[p], ke, hl, hg);
          const double re = hl - (Hs[p] - n.el[p]);
          s.e[p] = s.e[p] + (-re + s.V1[p]) / hg;
        }
        Hs[p] = Hs[p] + s.V1[p];
      }
      __syncthreads();
    }
    if (info == 0) {  // store the terminal state for the adjoint
      double* Wt = w.W + (size_t)b * n.nnzL;
      for (int t = threadIdx.x; t < n.nnzL; t += NT) Wt[t] = s.W[t];
      for (int k = threadIdx.x; k < n.L; k += NT) {
        const double q = s.q[k];
        w.P[(size_t)b * n.L + k] = s.P[k];
        double dr = 0.0;
        const int st = s.S[k];
        const bool closed = st <= WDS_CLOSED || (n.flags[k] & WDS_F_ZERO_SPEED);
        if ((n.flags[k] & WDS_F_IS_PIPE) && !closed) {
          const double sgn = q < 0.0 ? -1.0 : 1.0, qa = q * sgn;
          const double hgr = n.hexp * rrow[k] * pow(fmax(qa, 1e-30), n.hexp - 1.0);
          if (hgr >= n.rqtol) dr = pow(qa, n.hexp) * sgn;
        }
        w.dr[(size_t)b * n.L + k] = dr;
      }
      for (int p = threadIdx.x; p < n.Nj; p += NT) {
        const double ke = kerow[n.jnode[p]];
        double hge = 1.0, dke = 0.0;
        if (ke > 0.0) {
          double hl;
          emitter_hl(n, s.e[p], ke, hl, hge);
          const double ea = fabs(s.e[p]);
          const double pw = pow(fmax(ea, 1e-30), n.qexp - 1.0);
          const double raw = n.qexp * fmax(ke, kCSMALL) * pw;
          dke = (raw < n.rqtol || ke < kCSMALL) ? 0.0 : pw * s.e[p];
        }
        w.emh[(size_t)b * n.Nj + p] = s.emh[p];
        w.hge[(size_t)b * n.Nj + p] = hge;
        w.dke[(size_t)b * n.Nj + p] = dke;
      }
      const int pc = n.npcv > 0 ? n.npcv : 1;
      for (int i = threadIdx.x; i < n.npcv; i += NT)
        w.act[(size_t)b * pc + i] = s.S[n.pcv_link[i]] == WDS_ACTIVE ? 1 : 0;
    }
    for (int p = threadIdx.x; p < n.Nj; p += NT) s.V1[p] = Hs[p];
    __syncthreads();
  }
  if (threadIdx.x == 0) w.valid[b] = (a.polish >= 0 && info == 0) ? 1 : 0;
  // ---- outputs
  double* hrow = a.head + (size_t)b * n.N;
  double* erow = a.emit + (size_t)b * n.N;
  for (int f = threadIdx.x; f < n.Nf; f += NT) {
    hrow[n.fnode[f]] = s.hf[f];
    erow[n.fnode[f]] = 0.0;
  }
  for (int p = threadIdx.x; p < n.Nj; p += NT) {
    const int nd = n.jnode[p];
    hrow[nd] = s.V1[p];
    erow[nd] = kerow[nd] > 0.0 ? s.e[p] : 0.0;
  }
  for (int k = threadIdx.x; k < n.L; k += NT) {
    a.flow[(size_t)b * n.L + k] = s.q[k];
    a.status[(size_t)b * n.L + k] = s.S[k];
  }
  if (threadIdx.x == 0) {
    a.iters[b] = iters;
    a.relerr[b] = relerr;
    a.info[b] = info;
  }
}

// ---------------------------------------------------------------- adjoint kernel
// Node adjoint with constraint rows (autodiff.py:1107-1154) and the
// theta contraction (autodiff.py:1246-1312).
template <int NT>
__global__ void __launch_bounds__(NT) k_adjoint(DevNet n, DevWork w, AdjArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int b = blockIdx.x;
  Sh s = carve(n, smem_raw);
  if (!w.valid[b]) return;  // uniform per CTA
  const double* Wt = w.W + (size_t)b * n.nnzL;
  for (int t = threadIdx.x; t < n.nnzL; t += NT) s.W[t] = Wt[t];
  for (int k = threadIdx.x; k < n.L; k += NT) s.P[k] = w.P[(size_t)b * n.L + k];
  const int pc = n.npcv > 0 ? n.npcv : 1;
  // status is only consulted for ACTIVE flags of PRVs
  for (int k = threadIdx.x; k < n.L; k += NT) {
    const int i = n.link_pcv[k];
    s.S[k] = (i >= 0 && w.act[(size_t)b * pc + i]) ? WDS_ACTIVE : WDS_OPEN;
  }
  for (int p = threadIdx.x; p < n.Nj; p += NT) s.emh[p] = w.emh[(size_t)b * n.Nj + p];
  __syncthreads();
  const double* gH = a.gH + (size_t)b * n.N;
  const double* gQ = a.gQ + (size_t)b * n.L;
  const double* gE = a.gE + (size_t)b * n.N;
  // r = B^T P gQ - em gE / hge - gH
  for (int p = threadIdx.x; p < n.Nj; p += NT) {
    const int a0 = n.inc_ptr[p], m = n.inc_split[p], z = n.inc_ptr[p + 1];
    double acc = 0.0;
    for (int e = m; e < z; ++e) {
      const int k = n.inc[e];
      acc += s.P[k] * gQ[k];
    }
    for (int e = a0; e < m; ++e) {
      const int k = n.inc[e];
      acc += -(s.P[k] * gQ[k]);
    }
    const int nd = n.jnode[p];
    s.V0[p] = (acc - s.emh[p] * gE[nd]) - gH[nd];
  }
  bool any_act = false;
  for (int i = threadIdx.x; i < n.npcv; i += NT) any_act |= s.S[n.pcv_link[i]] == WDS_ACTIVE;
  any_act = __syncthreads_or(any_act);
  double* lam = s.V1;
  double* t = s.V2;
  if (!any_act) {
    solve_refined<NT>(n, s.W, s.P, s.emh, s.S, s.V0, lam, t, 2);
  } else {
    const int p = n.npcv;
    double* scr = w.scr + (size_t)b * w.nscr * n.Nj;
    double* r2 = scr;
    double* res = r2 + n.Nj;
    double* sx = res + n.Nj;
    double* cols = sx + n.Nj;
    double* C = s.small;
    double* y = C + p * p;
    double* actf = y + p;
    if (threadIdx.x == 0)
      for (int i = 0; i < p; ++i) actf[i] = s.S[n.pcv_link[i]] == WDS_ACTIVE ? 1.0 : 0.0;
    for (int q = threadIdx.x; q < n.Nj; q += NT) r2[q] = s.V0[q];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < p; ++i)
        if (actf[i] != 0.0) r2[n.pcv_j2[i]] = gQ[n.pcv_link[i]];
    __syncthreads();
    solve_refined<NT>(n, s.W, s.P, s.emh, s.S, r2, lam, t, 2);
    for (int c = 0; c < p; ++c) {
      for (int q = threadIdx.x; q < n.Nj; q += NT) res[q] = q == n.pcv_j2[c] ? 1.0 : 0.0;
      __syncthreads();
      solve_refined<NT>(n, s.W, s.P, s.emh, s.S, res, cols + (size_t)c * n.Nj, t, 2);
    }
    if (threadIdx.x == 0)
      for (int a0 = 0; a0 < p; ++a0)
        for (int c = 0; c < p; ++c) {
          const double cw = cols[(size_t)c * n.Nj + n.pcv_j2[a0]] - cols[(size_t)c * n.Nj + n.pcv_j1[a0]];
          C[a0 * p + c] = cw * actf[a0] * actf[c] + (a0 == c ? 1.0 - actf[a0] : 0.0);
        }
    __syncthreads();
    auto wood = [&](double* x, const double* rr) {
      if (threadIdx.x == 0) {
        double Cc[64];
        for (int i = 0; i < p * p; ++i) Cc[i] = C[i];
        for (int a0 = 0; a0 < p; ++a0)
          y[a0] = (x[n.pcv_j2[a0]] - x[n.pcv_j1[a0]] - rr[n.pcv_j2[a0]]) * actf[a0];
        dense_solve(Cc, y, p);
      }
      __syncthreads();
      for (int q = threadIdx.x; q < n.Nj; q += NT) {
        double acc = 0.0;
        for (int c = 0; c < p; ++c) acc += cols[(size_t)c * n.Nj + q] * y[c];
        x[q] = x[q] - acc;
      }
      __syncthreads();
    };
    wood(lam, r2);
    for (int it = 0; it < 2; ++it) {
      for (int q = threadIdx.x; q < n.Nj; q += NT) res[q] = r2[q] - amul_node(n, q, s.P, lam, s.emh, s.S);
      __syncthreads();
      if (threadIdx.x == 0)
        for (int i = 0; i < p; ++i)
          if (actf[i] != 0.0)
            res[n.pcv_j2[i]] = r2[n.pcv_j2[i]] - (lam[n.pcv_j2[i]] - lam[n.pcv_j1[i]]);
      __syncthreads();
      solve_refined<NT>(n, s.W, s.P, s.emh, s.S, res, sx, t, 2);
      wood(sx, res);
      for (int q = threadIdx.x; q < n.Nj; q += NT) lam[q] = lam[q] + sx[q];
      __syncthreads();
    }
  }
  // theta contraction
  double* gd = a.gd + (size_t)b * n.N;
  double* gke = a.gke + (size_t)b * n.N;
  double* grh = a.grh + (size_t)b * n.N;
  double* gr = a.gr + (size_t)b * n.L;
  const double* hge = w.hge + (size_t)b * n.Nj;
  const double* dke = w.dke + (size_t)b * n.Nj;
  for (int p = threadIdx.x; p < n.Nj; p += NT) {
    const int nd = n.jnode[p];
    gd[nd] = lam[p];
    double g = 0.0;
    if (s.emh[p] != 0.0) {
      const double lam_e = (gE[nd] + lam[p]) / hge[p];
      g = -(lam_e * dke[p]);
    }
    gke[nd] = g;
    grh[nd] = 0.0;
  }
  const double* dr = w.dr + (size_t)b * n.L;
  for (int k = threadIdx.x; k < n.L; k += NT) {
    const double l1 = junc_of(n.e1[k], lam), l2 = junc_of(n.e2[k], lam);
    const double lam_l = s.P[k] * (gQ[k] - (l2 - l1));
    gr[k] = -(lam_l * dr[k]);
  }
  for (int f = threadIdx.x; f < n.Nf; f += NT) {
    const int nd = n.fnode[f];
    double acc = 0.0;
    for (int e = n.finc_ptr[f]; e < n.finc_split[f]; ++e) {
      const int k = n.finc[e];
      const double l1 = junc_of(n.e1[k], lam), l2 = junc_of(n.e2[k], lam);
      acc += s.P[k] * (gQ[k] - (l2 - l1));
    }
    for (int e = n.finc_split[f]; e < n.finc_ptr[f + 1]; ++e) {
      const int k = n.finc[e];
      const double l1 = junc_of(n.e1[k], lam), l2 = junc_of(n.e2[k], lam);
      acc += -(s.P[k] * (gQ[k] - (l2 - l1)));
    }
    grh[nd] = acc + gH[nd];
    gd[nd] = 0.0;
    gke[nd] = 0.0;
  }
}

size_t smem_bytes(const DevNet& n) {
  auto a16 = [](size_t x) { return (x + 15) / 16 * 16; };
  size_t o = 0;
  o += 3 * a16(8ull * n.L);
  o += a16(8ull * n.nnzL);
  o += 5 * a16(8ull * n.Nj);
  o += a16(8ull * (n.Nf > 0 ? n.Nf : 1));
  o += a16(8ull * (n.nxf > 0 ? n.nxf : 1));
  o += a16(8ull * 4 * 32);
  o += a16(8ull * (4 * n.npcv * n.npcv + 5 * n.npcv + 8));
  o += a16(n.L);
  return o;
}

}  // namespace

size_t forward_smem_bytes(const DevNet& n, int) { return smem_bytes(n); }
size_t adjoint_smem_bytes(const DevNet& n, int) { return smem_bytes(n); }

int launch_forward(const DevNet& n, const DevWork& w, const FwdArgs& a, size_t smem, int threads,
                   void* stream, std::string* err) {
  if (n.npcv > 4) {
    *err = "wds_forward: more than 4 status-machine PRVs is not supported by this build";
    return WDS_E_UNSUPPORTED;
  }
  auto kern = k_forward<256>;
  cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (ce != cudaSuccess) {
    *err = std::string("wds_forward: ") + cudaGetErrorString(ce);
    return WDS_E_CUDA;
  }
  kern<<<a.B, 256, smem, (cudaStream_t)stream>>>(n, w, a);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("wds_forward launch: ") + cudaGetErrorString(ce);
    return WDS_E_CUDA;
  }
  return WDS_OK;
}

int launch_adjoint(const DevNet& n, const DevWork& w, const AdjArgs& a, size_t smem, int threads,
                   void* stream, std::string* err) {
  if (n.npcv > 4) {
    *err = "wds_adjoint: more than 4 status-machine PRVs is not supported by this build";
    return WDS_E_UNSUPPORTED;
  }
  auto kern = k_adjoint<256>;
  cudaError_t ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (ce != cudaSuccess) {
    *err = std::string("wds_adjoint: ") + cudaGetErrorString(ce);
    return WDS_E_CUDA;
  }
  kern<<<a.B, 256, smem, (cudaStream_t)stream>>>(n, w, a);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("wds_adjoint launch: ") + cudaGetErrorString(ce);
    return WDS_E_CUDA;
  }
  return WDS_OK;
}

}  // namespace wds
