// Device code of the fused batched GGA forward and reduced implicit adjoint
// for sm_100a.  Included by the kernel-instance sources (wds_k_*.cu), each of
// which instantiates one kernel kind in one factor precision, so that the
// instances compile in parallel; the launchers (wds_launch.cu) reach them
// through the kernel selectors at the end of this file.
//
// A CTA holds `GR` independent scenario groups of 256 threads.  Each group owns
// one scenario at a time: its link flows and coefficients, the LDL^T factor of
// the node matrix and the node vectors live in shared memory from the first
// Newton iteration to the terminal factorisation, so there is no host round
// trip inside the loop.  The symbolic schedule (update lists, row and column
// structure, incidence lists) is staged once per CTA into shared memory as
// 16-bit tables and shared by the groups.  Groups synchronise on their own
// named barriers, so they advance independently.
//
// Per GGA iteration (dgga/solver.py:2922-3179):
//   link pass    P, Y from the headloss formulas (one thread per link)
//   node pass    gather assembly of A (diagonal, pairs) and F in the
//                reference's scatter order; PRV valve coefficients after the
//                node coefficients (serial over the few PRVs)
//   factor       left-looking LDL^T, dependency-driven: a column starts as soon
//                as the columns it depends on are done (shared-memory counters)
//   solve        dependency-driven forward/backward substitution + refinement
//                against the matrix-free operator A x
//   update       dq = Y - P dh, emitter update, relerr reduction, status
//                machine (valve status every iteration, link status on the
//                converged / periodic branches, per-scenario nextcheck)
// Implicit mode then runs the reduced Newton polish with Woodbury row
// replacement for ACTIVE PRVs (dgga/autodiff.py:965-1104) and stores the
// terminal factor and coefficients for the adjoint kernel.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <algorithm>
#include <type_traits>

#include "wds_internal.h"

namespace wds {
namespace {

constexpr double kINF = __builtin_huge_val();
// A polish step keeps the factor in use while every link conductance P and
// emitter term of the step is within kReuseStep (relative) of the values it
// was factored with; the terminal state kept for the adjoint, within
// kReuseTerminal.
constexpr double kReuseStep = 1e-3;
constexpr double kReuseTerminal = 1e-4;
// ... and only once the previous step moved the flows by at most this
// fraction (sum |dq| / sum |q|): the polish is then in its quadratic regime,
// where a chord step equals the Newton step to rounding.
constexpr double kReuseFlow = 1e-6;

struct Sh {
  double *q, *P, *Y, *W, *V0, *V1, *V2, *hf, *xf, *red, *small;
  float* Wf;                      // the factor when it is kept in FP32 (W is then null)
  double *em_e, *em_ke, *em_emh;  // per emitter slot: flow, coefficient, 1/hgrad
  int16_t* eslot;                 // [Nj] emitter slot of a junction or -1
  double* tb;                     // [2][49] pivot columns (+ 1/pivot) of the top-block inversion
  double* Mg;                     // [nT][nT] top-block inverse (global workspace)
  int *wcnt, *flag, *err;
  int8_t* S;
};

// View of the compact schedule tables.  Slot-valued tables (positions in the
// factor W, in the update-term list and in the row lists) hold Slot: uint16_t
// for networks whose tables fit 16 bits (staged into shared memory), uint32_t
// for large networks (tables read from global memory).  Junction, link and
// incidence indices are 16-bit in both.
template <class Slot>
struct TabT {
  static constexpr bool kWide = sizeof(Slot) == 4;
  const uint32_t* spair;      // per slot: begin | count << 16 | diagonal << 31 (wide: 2 words, begin and count | diagonal << 31)
  const Slot* fpair;          // [3 * terms] {slot L_ik, slot L_jk, slot 1/D_k}
  const Slot* colptr;         // [Nj+1]
  const uint16_t* rowidx;     // [nnzL]
  const uint16_t* levptr;     // [nlev+1] columns of a level (columns numbered in level order)
  const Slot* rptr;           // [Nj+1] row lists
  const uint32_t* rent;       // row entries slot | k << 16 (wide: 2 words, slot and k)
  const uint8_t* mfac;        // [nlev] mode: log2 G | wide << 7
  const uint8_t* mfwd;
  const uint8_t* mbwd;
  const uint16_t* inc_ptr;    // [Nj+1]
  const uint16_t* inc_split;  // [Nj]
  const uint32_t* inc;        // link | PRV << 16 | other fixed << 17 | fixed index << 18
  const int16_t* e1;          // [L] end codes
  const int16_t* e2;
  const uint16_t* pptr;       // [npairs+1]
  const uint16_t* plink;      // link | PRV << 15
  const Slot* pslot;          // [npairs]
  const Slot* fill;           // [nfill]
  const Slot* dslot;          // [nT (nT+1) / 2] slot of top-block entry (i >= j) or all ones

  // update list of the entry in `slot`: first term, term count, diagonal flag
  __device__ __forceinline__ void sp(int slot, int& pb, int& cnt, bool& diag) const {
    if constexpr (kWide) {
      const uint2 w = reinterpret_cast<const uint2*>(spair)[slot];
      pb = (int)w.x;
      cnt = (int)(w.y & 0x7fffffffu);
      diag = (w.y >> 31) != 0;
    } else {
      const uint32_t w = spair[slot];
      pb = (int)(w & 0xffffu);
      cnt = (int)((w >> 16) & 0x7fffu);
      diag = (w >> 31) != 0;
    }
  }
  // row-list entry e: slot of L_jk and column k
  __device__ __forceinline__ void re(int e, int& slot, int& k) const {
    if constexpr (kWide) {
      const uint2 w = reinterpret_cast<const uint2*>(rent)[e];
      slot = (int)w.x;
      k = (int)w.y;
    } else {
      const uint32_t w = rent[e];
      slot = (int)(w & 0xffffu);
      k = (int)(w >> 16);
    }
  }
  __device__ __forceinline__ int cp(int j) const { return (int)colptr[j]; }
};
using STab = TabT<uint16_t>;
using LTab = TabT<uint32_t>;

template <class TB>
__device__ TB tab_view(const DevNet& n, const unsigned char* b) {
  using Slot = typename std::remove_pointer<decltype(TB::colptr)>::type;
  using S = typename std::remove_const<Slot>::type;
  TB t;
  t.spair = (const uint32_t*)(b + n.o_spair);
  t.fpair = (const S*)(b + n.o_fpair);
  t.colptr = (const S*)(b + n.o_colptr);
  t.rowidx = (const uint16_t*)(b + n.o_rowidx);
  t.levptr = (const uint16_t*)(b + n.o_levptr);
  t.rptr = (const S*)(b + n.o_rptr);
  t.rent = (const uint32_t*)(b + n.o_rent);
  t.mfac = (const uint8_t*)(b + n.o_mode);
  t.mfwd = t.mfac + n.nlev;
  t.mbwd = t.mfwd + n.nlev;
  t.inc_ptr = (const uint16_t*)(b + n.o_inc_ptr);
  t.inc_split = (const uint16_t*)(b + n.o_inc_split);
  t.inc = (const uint32_t*)(b + n.o_inc);
  t.e1 = (const int16_t*)(b + n.o_e1);
  t.e2 = (const int16_t*)(b + n.o_e2);
  t.pptr = (const uint16_t*)(b + n.o_pptr);
  t.plink = (const uint16_t*)(b + n.o_plink);
  t.pslot = (const S*)(b + n.o_pslot);
  t.fill = (const S*)(b + n.o_fill);
  t.dslot = (const S*)(b + n.o_dslot);
  return t;
}

// link index of an incidence entry (the upper bits carry flags)
template <class TB>
__device__ __forceinline__ int inc_link(const TB& T, int e) { return (int)(T.inc[e] & 0xffffu); }

__device__ __forceinline__ double head_of(int c, const double* x, const double* hf) {
  return c >= 0 ? x[c] : hf[-c - 1];
}
__device__ __forceinline__ double junc_of(int c, const double* x) { return c >= 0 ? x[c] : 0.0; }

// ---------------------------------------------------------------- groups
// A group synchronises with its own named barrier (id 1 + group index).
template <int NT>
__device__ __forceinline__ int gtid() { return threadIdx.x & (NT - 1); }
// The warp of a group that runs the narrow levels: warp g mod 4 of group g,
// so that the co-resident groups' narrow chains issue from different SM
// sub-partitions (warp w of a CTA issues from sub-partition w mod 4).
template <int NT>
__device__ __forceinline__ bool in_narrow_warp() {
  constexpr int kWarps = NT / 32;
  const int g = (int)(threadIdx.x / NT) & 3;
  return (gtid<NT>() >> 5) == (g < kWarps ? g : 0);
}
template <int NT>
__device__ __forceinline__ void gsync() {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)(threadIdx.x / NT)), "r"(NT) : "memory");
}
template <int NT>
__device__ __forceinline__ bool gsync_or(bool p) {
  unsigned r;
  asm volatile(
      "{\n\t.reg .pred ip, op;\n\tsetp.ne.u32 ip, %1, 0;\n\t"
      "bar.red.or.pred op, %2, %3, ip;\n\tselp.u32 %0, 1, 0, op;\n\t}"
      : "=r"(r)
      : "r"((unsigned)p), "r"(1 + (int)(threadIdx.x / NT)), "r"(NT)
      : "memory");
  return r != 0;
}

// Deterministic group sum of m <= 4 values (warp butterflies, then a fixed
// order over the warps); every thread gets the same result.
template <int NT>
__device__ void block_sum(double* v, int m, double* red) {
  for (int i = 0; i < m; ++i)
    for (int o = 16; o; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
  const int w = gtid<NT>() >> 5, l = threadIdx.x & 31;
  gsync<NT>();
  if (l == 0)
    for (int i = 0; i < m; ++i) red[w * 4 + i] = v[i];
  gsync<NT>();
  for (int i = 0; i < m; ++i) {
    double s = 0.0;
    for (int ww = 0; ww < NT / 32; ++ww) s += red[ww * 4 + i];
    v[i] = s;
  }
}

// Group maximum of mx and minimum of mn (warp butterflies, then the warps'
// values in order); every thread gets both results.
template <int NT>
__device__ void block_maxmin(double& mx, double& mn, double* red) {
  for (int o = 16; o; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  }
  const int w = gtid<NT>() >> 5, l = threadIdx.x & 31;
  gsync<NT>();
  if (l == 0) {
    red[w * 4] = mx;
    red[w * 4 + 1] = mn;
  }
  gsync<NT>();
  for (int ww = 0; ww < NT / 32; ++ww) {
    mx = fmax(mx, red[ww * 4]);
    mn = fmin(mn, red[ww * 4 + 1]);
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

// Pump parameters of one scenario: rows of [L] values read at pump links
// (the network's own, or the call's speed / pump_h0 / pump_r of
// implicit_solve, dgga/autodiff.py:1315-1342), read through the kernel
// arguments only where a pump needs them.  own_sp: the speeds are the call's,
// so the zero-speed and pumpstatus tests are taken from them instead of the
// network's link flags.
struct PumpTh {
  const FwdArgs& a;
  const DevNet& n;
  long long o;  // row offset of this scenario
  __device__ __forceinline__ bool own_sp() const { return a.th_sp != nullptr; }
  __device__ __forceinline__ double sp(int k) const { return a.th_sp ? a.th_sp[o + k] : n.pspeed[k]; }
  __device__ __forceinline__ double h0(int k) const { return a.th_h0 ? a.th_h0[o + k] : n.ph0[k]; }
  __device__ __forceinline__ double r(int k) const { return a.th_r ? a.th_r[o + k] : n.pr[k]; }
};

__device__ __forceinline__ PumpTh pump_th(const DevNet& n, const FwdArgs& a, int b) {
  return PumpTh{a, n, (long long)b * a.th_stride};
}

// A pump on the closed branch for its speed alone (hydcoeffs.c:696-701 via
// dgga/solver.py:673: setting == 0).
__device__ __forceinline__ bool zero_speed(const DevNet& n, const PumpTh& th, int k, int kd) {
  return th.own_sp() ? (kd == WDS_KIND_PUMP && th.sp(k) == 0.0)
                     : (n.flags[k] & WDS_F_ZERO_SPEED) != 0;
}

// pumpcoeff for every curve kind (dgga/solver.py:2221-2326)
__device__ void pump_coef(const DevNet& n, const PumpTh& th, int k, double q, double& P,
                          double& Y) {
  const int t = n.ptype[k];
  if (t == 3) {  // NOCURVE: an open valve
    P = 1.0 / kCSMALL;
    Y = q;
    return;
  }
  const double sgn = q < 0.0 ? -1.0 : 1.0;
  const double qa = q * sgn;
  const double spc = fmax(th.sp(k), 1e-12);
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
    const double h0e = spc * spc * th.h0(k);
    const double re = th.r(k) * pow(spc, 2.0 - pn);
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

// Coefficients of a control valve that is not ACTIVE (valvecoeff, as
// restated in dgga/solver.py:862-903 and _valvecoeff_scalar): CLOSED is the
// 1/CBIG branch, otherwise the minor-loss Km (or 1/CSMALL for Km = 0).
__device__ __forceinline__ void valve_state_coef(const DevNet& n, double km, double qk, int sk,
                                                 double& P, double& Y) {
  const bool cl = sk <= WDS_CLOSED;
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
  P = cl ? 1.0 / kCBIG : po;
  Y = cl ? qk : yo;
}

// PRV valve coefficients of one status-machine PRV (dgga/solver.py:862-903):
// returns pna (the non-ACTIVE P, zero when ACTIVE) and yna.
__device__ __forceinline__ void prv_open(const DevNet& n, int i, double qk, int sk, double& pna,
                                         double& yna) {
  double P;
  valve_state_coef(n, n.pcv_km[i], qk, sk, P, yna);
  pna = P * (sk == WDS_ACTIVE ? 0.0 : 1.0);
}

// Link coefficients of the headloss stage (dgga/solver.py:2923-2956).
// `adj` selects the adjoint/polish variant in which a status-machine PRV
// takes its valve coefficients directly (autodiff.py:838-847).
__device__ __forceinline__ void link_coef(const DevNet& n, const PumpTh& th, int k, double q,
                                          int s, double r, bool adj, double& P, double& Y) {
  const int kd = n.kind[k];
  if (kd == WDS_KIND_FCV) {  // the valve pass fills the GGA coefficients
    if (!adj) {
      P = 0.0;
      Y = 0.0;
    } else if (s == WDS_ACTIVE) {  // hloss = CBIG (q - qset), hgrad = CBIG
      P = 1.0 / kCBIG;
      Y = q - n.fcv_qs[n.link_fcv[k]];
    } else {
      valve_state_coef(n, n.fcv_km[n.link_fcv[k]], q, s, P, Y);
    }
    return;
  }
  if (kd == WDS_KIND_PRV || kd == WDS_KIND_PSV) {
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
  if (s <= WDS_CLOSED || zero_speed(n, th, k, kd)) {
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
    pump_coef(n, th, k, q, P, Y);
}

// d hloss / d(speed, H0, R) of one open pump at flow q with the curve
// segment / clamp branch frozen (dgga/autodiff.py:122-218, the CPU adjoint's
// pump theta; hydcoeffs.c:673-791).  Zero on the closed, zero-speed, NOCURVE
// and clamped constant-HP branches.
__device__ void pump_dtheta(const DevNet& n, const PumpTh& th, int k, double q, int st,
                            double& dw, double& dh0, double& dR) {
  dw = dh0 = dR = 0.0;
  const double w = th.sp(k);
  const int t = n.ptype[k];
  if (st <= WDS_CLOSED || w == 0.0 || t == 3) return;
  const double qa = fabs(q);
  if (t == 2) {  // CUSTOM: dw = 2 w H0c + Rc q on the frozen segment
    const int c0 = n.cptr[k], np = n.cptr[k + 1] - c0;
    const double* X = n.cx + c0;
    const double* Yc = n.cy + c0;
    const double spc = fmax(w, 1e-12);
    const double qq = (qa / spc) * n.ucf_flow;
    int idx = 0;
    while (idx < np && X[idx] < qq) ++idx;
    const int k2 = min(max(idx, 1), np - 1), k1 = k2 - 1;
    double rc = (Yc[k2] - Yc[k1]) / (X[k2] - X[k1]);
    double h0c = Yc[k1] - rc * X[k1];
    h0c = h0c / n.ucf_head;
    rc = rc * n.ucf_flow / n.ucf_head;
    dw = 2.0 * w * (-h0c) + (-rc) * q;
    return;
  }
  const double pn = n.pn[k], H0 = th.h0(k), R = th.r(k);
  if (t == 0) {  // CONST_HP: hloss = r / q on the unclamped branch only
    const double r = R * pow(w, 2.0 - pn);
    const double hgr = qa > 0.0 ? -r / qa / qa : kINF;
    if (hgr > kCBIG || hgr < n.rqtol) return;
    dw = (2.0 - pn) * R * pow(w, 1.0 - pn) / q;
    dR = pow(w, 2.0 - pn) / q;
    return;
  }
  dh0 = w * w;
  if (pn == 1.0) {  // linear curve
    dw = 2.0 * w * H0 + R * q;
    dR = w * q;
    return;
  }
  const double nm1 = pn - 1.0;
  const double pw = qa == 0.0 ? (nm1 > 0.0 ? 0.0 : (nm1 < 0.0 ? kINF : 1.0)) : pow(qa, nm1);
  const double hgr = pn * (R * pow(w, 2.0 - pn)) * pw;
  if (hgr < n.rqtol) {  // RQtol clamp: hloss = h0 + RQtol q
    dw = 2.0 * w * H0;
    return;
  }
  dw = 2.0 * w * H0 + (2.0 - pn) * R * pow(w, 1.0 - pn) * pw * q;
  dR = pow(w, 2.0 - pn) * pw * q;
}

// ---------------------------------------------------------------- linear algebra
// Matrix-free (A x)_p of the node matrix: links with conductance P, emitter
// diagonal emh, CBIG on the downstream node of ACTIVE PRVs
// (dgga/autodiff.py:878-895; the same operator the forward assembles).
template <class TB>
__device__ __forceinline__ double amul_node(const DevNet& n, const TB& T, const Sh& s, int p,
                                            const double* x) {
  const double* P = s.P;
  const int8_t* S = s.S;
  double acc = 0.0;
  const int a = T.inc_ptr[p], m = T.inc_split[p], z = T.inc_ptr[p + 1];
  for (int e = a; e < m; ++e) {
    const int k = inc_link(T, e);
    acc += P[k] * (junc_of(T.e1[k], x) - junc_of(T.e2[k], x));
  }
  for (int e = m; e < z; ++e) {
    const int k = inc_link(T, e);
    acc += -(P[k] * (junc_of(T.e1[k], x) - junc_of(T.e2[k], x)));
  }
  const int es = s.eslot[p];
  acc = acc + (es >= 0 ? s.em_emh[es] : 0.0) * x[p];
  for (int c = n.cb_ptr[p]; c < n.cb_ptr[p + 1]; ++c) {
    const int i = n.cb_idx[c];
    const double act = S[n.pcv_link[i]] == WDS_ACTIVE ? 1.0 : 0.0;
    acc += x[p] * act * kCBIG;
  }
  return acc;
}

// Sum over a lane group of size 1 << lg (aligned groups inside a warp); every
// lane of the warp calls it with the same lg.
template <class FT>
__device__ __forceinline__ FT group_sum(FT v, int lg) {
  for (int o = (1 << lg) >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// The factor of the scenario in its storage precision FT (double, or float
// for the FP32 factor with FP64 refinement).
template <class FT>
__device__ __forceinline__ FT* wp(const Sh& s);
template <>
__device__ __forceinline__ double* wp<double>(const Sh& s) { return s.W; }
template <>
__device__ __forceinline__ float* wp<float>(const Sh& s) { return s.Wf; }

// Factor slots [t0, t1) (one level, or the Schur-complement step of the top
// block) on `nthr` threads (thread index t): the entries are split over lane
// groups of 1 << lg, each group reducing its entry's update list with warp
// shuffles.  Diagonal entries of factored columns become 1/D.
template <class TB, class FT>
__device__ __forceinline__ void fac_range(const TB& T, FT* W, int t0, int t1, int lg, int t,
                                          int nthr, bool& bad) {
  const int G = 1 << lg, li = t & (G - 1), per = nthr >> lg;
  for (int base = t0; base < t1; base += per) {
    const int slot = base + (t >> lg);
    const bool valid = slot < t1;
    bool diag = false;
    FT acc = 0;
    if (valid) {
      int pb, cnt;
      T.sp(slot, pb, cnt, diag);
      const int pe = pb + cnt;
      for (int pr = pb + li; pr < pe; pr += G) {
        const auto* f = T.fpair + 3 * pr;
        acc += W[f[0]] * W[f[1]] * W[f[2]];
      }
    }
    acc = group_sum(acc, lg);
    if (valid && li == 0) {
      const FT w = W[slot] - acc;
      if (diag) {
        if (!(w > FT(0)) || !isfinite(w)) bad = true;
        W[slot] = FT(1) / w;
      } else {
        W[slot] = w;
      }
    }
  }
}

// Forward substitution over rows [c0, c1): v_j = (v_j - sum_k L_jk D_k u_k) / D_j,
// or, for the rows of the top block (top), v_j = v_j - sum over the lower columns.
template <class TB, class FT>
__device__ __forceinline__ void fwd_range(const TB& T, const FT* W, double* v, int c0,
                                          int c1, int lg, int t, int nthr, bool top) {
  const int G = 1 << lg, li = t & (G - 1), per = nthr >> lg;
  for (int base = c0; base < c1; base += per) {
    const int j = base + (t >> lg);
    const bool valid = j < c1;
    FT acc = 0;
    if (valid) {
      const int e1 = (int)T.rptr[j + 1];
      for (int e = (int)T.rptr[j] + li; e < e1; e += G) {
        int sl, k;
        T.re(e, sl, k);
        acc += W[sl] * (FT)v[k];
      }
    }
    acc = group_sum(acc, lg);
    if (valid && li == 0) {
      const FT vj = (FT)v[j];
      v[j] = (double)(top ? vj - acc : (vj - acc) * W[T.colptr[j]]);
    }
  }
}

// One backward-substitution level, columns [c0, c1):
// x_j = u_j - (1/D_j) sum_i L_ij D_j x_i.
template <class TB, class FT>
__device__ __forceinline__ void bwd_level(const TB& T, const FT* W, double* v, int c0, int c1,
                                          int lg, int t, int nthr) {
  const int G = 1 << lg, li = t & (G - 1), per = nthr >> lg;
  for (int base = c0; base < c1; base += per) {
    const int j = base + (t >> lg);
    const bool valid = j < c1;
    int cb = 0;
    FT acc = 0;
    if (valid) {
      cb = T.colptr[j];
      const int ce = T.colptr[j + 1];
      for (int e = cb + 1 + li; e < ce; e += G) acc += W[e] * (FT)v[T.rowidx[e]];
    }
    acc = group_sum(acc, lg);
    if (valid && li == 0) v[j] = (double)((FT)v[j] - W[cb] * acc);
  }
}

// 2^-h with h = ceil(e / 2) for x = m 2^e (m in [1, 2)), so that x 2^-2h lies
// in [0.5, 2); 1 for a diagonal that is not positive and finite (the pivot
// check then reports it).  Scaling by it is exact.
__device__ __forceinline__ double pow2_scale(double x) {
  if (!(x > 0.0) || !isfinite(x)) return 1.0;
  const long long e = ((__double_as_longlong(x) >> 52) & 0x7ff) - 1023;
  const long long h = (e + 1) >> 1;
  return __longlong_as_double((1023 - h) << 52);
}

// One sweep of the top-block inversion (see top_inverse) for pivot k, which
// lies in register block KB; NJ is the register block of column k + 1 and PAR
// the parity of k (the buffer that holds column k).  All three are static,
// so that no register is selected at run time.
template <int NT, int KB, int NJ, int PAR>
__device__ __forceinline__ void top_sweep(int k, int nT, int r, int c, double (&a)[3][3],
                                          double* tb, int& bad) {
  constexpr int ST = WDS_TOP_MAX + 1;
  const double* cb = tb + PAR * ST;
  double* nb = tb + (1 - PAR) * ST;
  const double ip = cb[WDS_TOP_MAX];
  const double c0 = cb[c], c1 = cb[c + 16], c2 = cb[c + 32];
#pragma unroll
  for (int ia = 0; ia < 3; ++ia) {
    const double t = cb[r + 16 * ia] * ip;
    a[ia][0] = fma(-t, c0, a[ia][0]);
    a[ia][1] = fma(-t, c1, a[ia][1]);
    a[ia][2] = fma(-t, c2, a[ia][2]);
  }
  const int km = k & 15;
  if (r == km && c == km) a[KB][KB] = -ip;  // the pivot: a_kk = -1/p
  // publish column kn = k + 1 (all rows: the full matrix is kept), then
  // p - 1 at its pivot and 1/p
  const int kn = k + 1, kq = kn & 15;
  if (kn < nT && c == kq) {
    nb[r] = a[0][NJ];
    nb[r + 16] = a[1][NJ];
    nb[r + 32] = a[2][NJ];
    if (r == kq) {
      const double x = a[NJ][NJ];
      if (!(x > 0.0) || !isfinite(x)) bad = 1;
      nb[WDS_TOP_MAX] = __drcp_rn(x);
      nb[kn] = x - 1.0;
    }
  }
  gsync<NT>();
}

// The sweeps k in [16 KB, min(16 KB + 16, nT)): in pairs (static parity);
// column k + 1 lies in block KB except after the block's last pivot.
template <int NT, int KB>
__device__ __forceinline__ void top_block(int nT, int r, int c, double (&a)[3][3], double* tb,
                                          int& bad) {
  const int k0 = 16 * KB;
  if (k0 >= nT) return;
  const int kend = min(k0 + 16, nT), kmid = min(k0 + 15, kend);
  int k = k0;
#pragma unroll 1
  for (; k + 1 < kmid; k += 2) {
    top_sweep<NT, KB, KB, 0>(k, nT, r, c, a, tb, bad);
    top_sweep<NT, KB, KB, 1>(k + 1, nT, r, c, a, tb, bad);
  }
  if (k < kmid) top_sweep<NT, KB, KB, 0>(k, nT, r, c, a, tb, bad);
  if (k0 + 15 < kend) top_sweep<NT, KB, (KB < 2 ? KB + 1 : KB), 1>(k0 + 15, nT, r, c, a, tb, bad);
}

// Inverse of the top block's Schur complement S (nT x nT, nT <= WDS_TOP_MAX)
// by symmetric sweeps (Gauss-Jordan elimination without pivoting, in column
// order; every pivot is then a pivot of the LDL^T of S, so its sign is the
// positive-definiteness check).  S is first scaled to S' = D S D with D the
// power-of-two diagonal that brings diag(S') into [0.5, 2) (exact), so the
// pivots p of S' are at most about 2, and S^{-1} = D S'^{-1} D.
// Sweeping k maps a_kk -> -1/p, a_ik -> a_ik/p, a_kj -> a_kj/p and
// a_ij -> a_ij - (a_ik/p) a_kj; after all nT sweeps the matrix is -S'^{-1}.
// With the pivot's entry of the published column set to p - 1, the one
// rank-1 update a_ij -> a_ij - (c_i/p) c_j (c = column k) gives row and
// column k as well: c_i - (c_i/p)(p - 1) = c_i/p, without cancellation since
// |p - 1| <= 1 after the scaling; only a_kk is then overwritten (-1/p).
// Thread (r, c) of a 16 x 16 grid holds the entries (r + 16 a, c + 16 b),
// a, b < 3, of the full matrix in registers for all sweeps, so that a sweep
// is 6 shared loads, 3 multiplies and 9 FMAs per thread; the sweep's code is
// instantiated per register block and buffer parity (top_block), so the
// sweep is short: about 430 cycles alone against 530 with the block chosen
// at run time.  Column k+1 after sweep k goes through shared memory: two
// alternating buffers of 49 (the column, then 1/p of its pivot, which the
// pivot's owner computes and checks) and one group barrier per sweep.  S is
// read from the factor slots listed in dslot, S^{-1} is written to Mg
// (row-major, each entry by its owner).  Returns 1 when this thread owned a
// pivot that was not positive and finite.  Runs as a separate function so
// that its block of registers does not add to the caller's.
template <int NT, class Slot, class FT>
__device__ __noinline__ int top_inverse(const FT* W, const Slot* dslot, double* tb,
                                        double* Mg, int nT) {
  static_assert(NT == 256 && WDS_TOP_MAX == 48, "16 x 16 threads x 3 x 3 entries");
  constexpr int ST = WDS_TOP_MAX + 1;
  const int tid = gtid<NT>(), r = tid >> 4, c = tid & 15;
  double a[3][3];
  int bad = 0;
#pragma unroll
  for (int ia = 0; ia < 3; ++ia)
#pragma unroll
    for (int jb = 0; jb < 3; ++jb) {
      const int i = r + 16 * ia, j = c + 16 * jb;
      double x = 0.0;
      if (i < nT && j < nT) {
        const int hi = i > j ? i : j, lo = i > j ? j : i;
        const Slot sl = dslot[hi * (hi + 1) / 2 + lo];
        if (sl != (Slot)~Slot(0)) x = (double)W[sl];
      }
      a[ia][jb] = x;
    }
  // the scale of row i goes through tb[ST + i] (the diagonal's owner writes it)
  if (r == c) {
#pragma unroll
    for (int ia = 0; ia < 3; ++ia)
      if (r + 16 * ia < nT) tb[ST + r + 16 * ia] = pow2_scale(a[ia][ia]);
  }
  gsync<NT>();
  double dr[3], dc[3];
#pragma unroll
  for (int ia = 0; ia < 3; ++ia) {
    dr[ia] = r + 16 * ia < nT ? tb[ST + r + 16 * ia] : 1.0;
    dc[ia] = c + 16 * ia < nT ? tb[ST + c + 16 * ia] : 1.0;
  }
#pragma unroll
  for (int ia = 0; ia < 3; ++ia)
#pragma unroll
    for (int jb = 0; jb < 3; ++jb) a[ia][jb] *= dr[ia] * dc[jb];
  gsync<NT>();
  // column 0 (rows beyond nT are zero), then p - 1 at the pivot and 1/p
  if (c == 0) {
#pragma unroll
    for (int ia = 0; ia < 3; ++ia) tb[r + 16 * ia] = a[ia][0];
    if (r == 0) {
      const double p = a[0][0];
      if (!(p > 0.0) || !isfinite(p)) bad = 1;
      tb[WDS_TOP_MAX] = __drcp_rn(p);
      tb[0] = p - 1.0;
    }
  }
  gsync<NT>();
  top_block<NT, 0>(nT, r, c, a, tb, bad);
  top_block<NT, 1>(nT, r, c, a, tb, bad);
  top_block<NT, 2>(nT, r, c, a, tb, bad);
#pragma unroll
  for (int ia = 0; ia < 3; ++ia)
#pragma unroll
    for (int jb = 0; jb < 3; ++jb) {
      const int i = r + 16 * ia, j = c + 16 * jb;
      if (i < nT && j < nT) Mg[i * nT + j] = -a[ia][jb] * (dr[ia] * dc[jb]);
    }
  return bad;
}

template <int NT>
__device__ __noinline__ void top_apply(const double* Mg, double* vT, int nT) {
  const int tid = gtid<NT>(), i = tid >> 2, li = tid & 3;
  double acc0 = 0.0, acc1 = 0.0;
  if (i < nT) {
    const double* row = Mg + i * nT;
#pragma unroll
    for (int q = 0; q < WDS_TOP_MAX / 4; q += 2) {
      const int j0 = li + 4 * q, j1 = j0 + 4;
      if (j0 < nT) acc0 += row[j0] * vT[j0];
      if (j1 < nT) acc1 += row[j1] * vT[j1];
    }
  }
  double acc = group_sum(acc0 + acc1, 2);
  gsync<NT>();
  if (i < nT && li == 0) vT[i] = acc;
  gsync<NT>();
}

// Level-scheduled LDL^T.  Wide levels (many independent entries) use all the
// group's threads and a group barrier; narrow levels run on warp 0 alone,
// separated by __syncwarp.  W holds A on entry (pattern of L, fill zero) and
// on exit the unscaled columns L_ij D_j with 1/D_j in the diagonal slot, for
// the columns below the top block; the top block's slots hold its Schur
// complement and its inverse goes to s.Mg.  Returns true when every pivot was
// positive and finite.
template <int NT, class FT, class TB>
__device__ bool factor(const DevNet& n, const TB& T, const Sh& s) {
  const int tid = gtid<NT>(), lane = tid & 31;
  const bool inw = in_narrow_warp<NT>();
  bool bad = false, prev_wide = true;
  // a level's mode and slot range are static: the next level's are loaded
  // while this level runs, so that a level starts with its own work
  int md_n = n.L0 > 0 ? T.mfac[0] : 0, t1_n = n.L0 > 0 ? T.colptr[T.levptr[1]] : 0;
  int t0 = 0;
  for (int lv = 0; lv < n.L0; ++lv) {
    const int md = md_n, t1 = t1_n;
    if (lv + 1 < n.L0) {
      md_n = T.mfac[lv + 1];
      t1_n = T.colptr[T.levptr[lv + 2]];
    }
    const bool wide = (md & 0x80) != 0;
    if (wide) {
      if (!prev_wide) gsync<NT>();
      fac_range(T, wp<FT>(s), t0, t1, md & 7, tid, NT, bad);
      gsync<NT>();
    } else if (inw) {
      fac_range(T, wp<FT>(s), t0, t1, md & 7, lane, 32, bad);
      __syncwarp();
    }
    prev_wide = wide;
    t0 = t1;
  }
  if (n.nT > 0) {
    // Schur complement of the top block: its slots minus the lower columns' updates
    const int md = T.mfac[n.L0];
    const int t0 = T.colptr[n.cT];
    if (!prev_wide) gsync<NT>();
    if (md & 0x80) fac_range(T, wp<FT>(s), t0, n.nnzL, md & 7, tid, NT, bad);
    else if (inw) fac_range(T, wp<FT>(s), t0, n.nnzL, md & 7, lane, 32, bad);
    gsync<NT>();
    if (top_inverse<NT>((const FT*)wp<FT>(s), T.dslot, s.tb, s.Mg, n.nT)) bad = true;
  }
  return !gsync_or<NT>(bad);
}

// In-place (L D L^T) v = b: forward levels below the top block, the top rows'
// right-hand side, the dense top solve, backward levels below the top block.
template <int NT, class FT, class TB>
__device__ void solve(const DevNet& n, const TB& T, const Sh& s, double* v) {
  const int tid = gtid<NT>(), lane = tid & 31;
  const bool inw = in_narrow_warp<NT>();
  bool prev_wide = true;
  // each level's mode and column range come from registers loaded a level ahead
  int md_n = n.L0 > 0 ? T.mfwd[0] : 0, c1_n = n.L0 > 0 ? T.levptr[1] : 0;
  int c0 = 0;
  for (int lv = 0; lv < n.L0; ++lv) {
    const int md = md_n, c1 = c1_n;
    if (lv + 1 < n.L0) {
      md_n = T.mfwd[lv + 1];
      c1_n = T.levptr[lv + 2];
    }
    const bool wide = (md & 0x80) != 0;
    if (wide) {
      if (!prev_wide) gsync<NT>();
      fwd_range(T, (const FT*)wp<FT>(s), v, c0, c1, md & 7, tid, NT, false);
      gsync<NT>();
    } else if (inw) {
      fwd_range(T, (const FT*)wp<FT>(s), v, c0, c1, md & 7, lane, 32, false);
      __syncwarp();
    }
    prev_wide = wide;
    c0 = c1;
  }
  if (n.nT > 0) {
    const int md = T.mfwd[n.L0];
    if (!prev_wide) gsync<NT>();
    if (md & 0x80) fwd_range(T, (const FT*)wp<FT>(s), v, n.cT, n.Nj, md & 7, tid, NT, true);
    else if (inw) fwd_range(T, (const FT*)wp<FT>(s), v, n.cT, n.Nj, md & 7, lane, 32, true);
    gsync<NT>();
    top_apply<NT>(s.Mg, v + n.cT, n.nT);
    prev_wide = true;
  }
  int mb_n = n.L0 > 0 ? T.mbwd[n.L0 - 1] : 0, b0_n = n.L0 > 0 ? T.levptr[n.L0 - 1] : 0;
  int b1 = n.L0 > 0 ? T.levptr[n.L0] : 0;
  for (int lv = n.L0 - 1; lv >= 0; --lv) {
    const int md = mb_n, b0 = b0_n;
    if (lv > 0) {
      mb_n = T.mbwd[lv - 1];
      b0_n = T.levptr[lv - 1];
    }
    const bool wide = (md & 0x80) != 0;
    if (wide) {
      if (!prev_wide) gsync<NT>();
      bwd_level(T, (const FT*)wp<FT>(s), v, b0, b1, md & 7, tid, NT);
      gsync<NT>();
    } else if (inw) {
      bwd_level(T, (const FT*)wp<FT>(s), v, b0, b1, md & 7, lane, 32);
      __syncwarp();
    }
    prev_wide = wide;
    b1 = b0;
  }
  gsync<NT>();
}

// x = A^{-1} rhs with `refine` refinement steps against the matrix-free A.
// unit >= 0 means rhs = e_unit.  An unrefined solve whose x lies outside
// shared memory (the Woodbury columns and refinement corrections in the
// global workspace) runs in the shared temporary t and stores x once, so
// that its substitution levels chain on shared-memory latency.
template <int NT, class FT, class TB>
__device__ void solve_refined(const DevNet& n, const TB& T, const Sh& s, const double* rhs,
                              int unit, double* x, double* t, int refine) {
  const int tid = gtid<NT>();
  const bool via_t = refine == 0 && t != nullptr && !__isShared(x) && __isShared(t);
  double* v = via_t ? t : x;
  for (int p = tid; p < n.Nj; p += NT) v[p] = unit >= 0 ? (p == unit ? 1.0 : 0.0) : rhs[p];
  gsync<NT>();
  solve<NT, FT>(n, T, s, v);
  if (via_t) {
    for (int p = tid; p < n.Nj; p += NT) x[p] = v[p];
    gsync<NT>();
    return;
  }
  for (int it = 0; it < refine; ++it) {
    for (int p = tid; p < n.Nj; p += NT) {
      const double b = unit >= 0 ? (p == unit ? 1.0 : 0.0) : rhs[p];
      t[p] = b - amul_node(n, T, s, p, x);
    }
    gsync<NT>();
    solve<NT, FT>(n, T, s, t);
    for (int p = tid; p < n.Nj; p += NT) x[p] = x[p] + t[p];
    gsync<NT>();
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
// into W (pattern of L) and F = V0; Xflow saved for PRV downstream nodes.
template <int NT, class FT, class TB>
__device__ void assemble_gga(const DevNet& n, const TB& T, const Sh& s, const double* kerow,
                             const double* dj) {
  const int tid = gtid<NT>();
  for (int p = tid; p < n.Nj; p += NT) {
    const int a = T.inc_ptr[p], m = T.inc_split[p], z = T.inc_ptr[p + 1];
    // the junction's global values are requested before its incidence sums
    const double dem = dj[p];
    const int xfs = n.node_xf[p];
    double dg = 0.0, xf = 0.0, F = 0.0;
    // the link flows and Y live in L2: the first kPre incident links' values
    // are requested together, then summed in the reference's order (n1 side,
    // then n2 side); a junction with more links loads the rest one by one
    constexpr int kPre = 4;
    double qv[kPre], yv[kPre];
#pragma unroll
    for (int u = 0; u < kPre; ++u) {
      qv[u] = yv[u] = 0.0;
      if (a + u < z) {
        const int k = T.inc[a + u] & 0xffff;
        qv[u] = s.q[k];
        yv[u] = s.Y[k];
      }
    }
#pragma unroll
    for (int u = 0; u < kPre; ++u) {
      const int e = a + u;
      if (e >= m) break;
      const uint32_t ie = T.inc[e];
      if (ie & (1u << 16)) continue;
      dg += s.P[ie & 0xffff];
      xf += -qv[u];
      F += yv[u];
    }
    for (int e = a + kPre; e < m; ++e) {
      const uint32_t ie = T.inc[e];
      if (ie & (1u << 16)) continue;
      const int k = ie & 0xffff;
      dg += s.P[k];
      xf += -s.q[k];
      F += s.Y[k];
    }
#pragma unroll
    for (int u = 0; u < kPre; ++u) {
      const int e = a + u;
      if (e < m || e >= z) continue;
      const uint32_t ie = T.inc[e];
      if (ie & (1u << 16)) continue;
      dg += s.P[ie & 0xffff];
      xf += qv[u];
      F += -yv[u];
    }
    for (int e = (m > a + kPre ? m : a + kPre); e < z; ++e) {
      const uint32_t ie = T.inc[e];
      if (ie & (1u << 16)) continue;
      const int k = ie & 0xffff;
      dg += s.P[k];
      xf += s.q[k];
      F += -s.Y[k];
    }
    for (int e = m; e < z; ++e) {  // n1 end fixed: F[Row[n2]] += P*H[n1]
      const uint32_t ie = T.inc[e];
      if ((ie & (1u << 16)) || !(ie & (1u << 17))) continue;
      F += s.P[ie & 0xffff] * s.hf[ie >> 18];
    }
    for (int e = a; e < m; ++e) {  // n2 end fixed: F[Row[n1]] += P*H[n2]
      const uint32_t ie = T.inc[e];
      if ((ie & (1u << 16)) || !(ie & (1u << 17))) continue;
      F += s.P[ie & 0xffff] * s.hf[ie >> 18];
    }
    const int es = s.eslot[p];
    if (es >= 0) {
      double hl, hg;
      emitter_hl(n, s.em_e[es], s.em_ke[es], hl, hg);
      const double emh = 1.0 / hg;
      s.em_emh[es] = emh;
      dg = dg + emh;
      F = F + (hl + n.el[p]) / hg;
      xf = xf - s.em_e[es];
    }
    xf = xf - dem;
    F = F + xf;
    wp<FT>(s)[T.colptr[p]] = (FT)dg;
    s.V0[p] = F;
    if (xfs >= 0) s.xf[xfs] = xf;
  }
  for (int t = tid; t < n.npairs; t += NT) {
    double v = 0.0;
    for (int e = T.pptr[t]; e < T.pptr[t + 1]; ++e) {
      const int pl = T.plink[e];
      if (pl & 0x8000) continue;
      v += -s.P[pl];
    }
    wp<FT>(s)[T.pslot[t]] = (FT)v;
  }
  for (int t = tid; t < n.nfill; t += NT) wp<FT>(s)[T.fill[t]] = FT(0);
  gsync<NT>();
  if (tid == 0) {  // valvecoeffs after nodecoeffs, in valve order
    for (int v = 0; v < n.npcv + n.nfcv; ++v) {
      const int o = n.vord[v];
      if (o < 0) {  // FCV (fcvcoeff, hydcoeffs.c:1047-1097 as in dgga/solver.py:1665-1695)
        const int f = -1 - o, k = n.fcv_link[f];
        const double qk = s.q[k];
        const int j1 = n.fcv_j1[f], j2 = n.fcv_j2[f];
        FT* W = wp<FT>(s);
        double pk, yk;
        if (s.S[k] == WDS_ACTIVE) {
          // the setting cuts the network: an outflow at n1, an inflow at n2
          const double qs = n.fcv_qs[f];
          if (n.fcv_xf1[f] >= 0) s.xf[n.fcv_xf1[f]] -= qs;
          if (n.fcv_xf2[f] >= 0) s.xf[n.fcv_xf2[f]] += qs;
          yk = qk - qs;
          s.V0[j1] -= qs;
          s.V0[j2] += qs;
          pk = 1.0 / kCBIG;
        } else {
          valve_state_coef(n, n.fcv_km[f], qk, s.S[k], pk, yk);
          s.V0[j1] += yk - qk;
          s.V0[j2] -= yk - qk;
        }
        W[n.fcv_off[f]] += (FT)(-pk);
        W[T.colptr[j1]] += (FT)pk;
        W[T.colptr[j2]] += (FT)pk;
        s.P[k] = pk;
        s.Y[k] = yk;
        continue;
      }
      const int i = o;
      const int k = n.pcv_link[i];
      const double qk = s.q[k];
      const int sk = s.S[k];
      const bool act = sk == WDS_ACTIVE;
      double pna, yna;
      prv_open(n, i, qk, sk, pna, yna);
      const double mna = act ? 0.0 : 1.0, mact = act ? 1.0 : 0.0;
      // prvcoeff / psvcoeff (hydcoeffs.c:959-1044 as in dgga/solver.py:
      // 862-903, 1647-1664): an ACTIVE valve holds the head of jc (PRV: n2,
      // PSV: n1) by a CBIG penalty and reads the flow excess there
      const double xfc = s.xf[n.pcv_xf[i]], sg = n.pcv_sgn[i];
      const double dy = (yna - qk) * mna;
      const int j1 = n.pcv_j1[i], j2 = n.pcv_j2[i], jc = n.pcv_jc[i], jo = n.pcv_jo[i];
      const double fo = (act && sg * xfc < 0.0) ? xfc : 0.0;
      FT* W = wp<FT>(s);
      W[n.pcv_off[i]] += (FT)(-pna);
      W[T.colptr[j1]] += (FT)pna;
      W[T.colptr[j2]] += (FT)pna;
      W[T.colptr[jc]] += (FT)(kCBIG * mact);
      s.V0[j1] += dy;
      s.V0[j2] -= dy;
      s.V0[jo] += fo;
      s.V0[jc] += n.pcv_hset[i] * kCBIG * mact;
      s.P[k] = pna;
      s.Y[k] = act ? qk + sg * xfc : yna;
    }
  }
  gsync<NT>();
}

// Reduced-matrix assembly at the current state (dgga/autodiff.py:928-962):
// every link with its P, + emh diagonal, + CBIG on ACTIVE PRV downstream nodes.
template <int NT, class FT, class TB>
__device__ void assemble_reduced(const DevNet& n, const TB& T, const Sh& s) {
  const int tid = gtid<NT>();
  for (int p = tid; p < n.Nj; p += NT) {
    double dg = 0.0;
    for (int e = T.inc_ptr[p]; e < T.inc_ptr[p + 1]; ++e) dg += s.P[inc_link(T, e)];
    const int es = s.eslot[p];
    dg = dg + (es >= 0 ? s.em_emh[es] : 0.0);
    for (int c = n.cb_ptr[p]; c < n.cb_ptr[p + 1]; ++c) {
      const int i = n.cb_idx[c];
      dg += kCBIG * (s.S[n.pcv_link[i]] == WDS_ACTIVE ? 1.0 : 0.0);
    }
    wp<FT>(s)[T.colptr[p]] = (FT)dg;
  }
  for (int t = tid; t < n.npairs; t += NT) {
    double v = 0.0;
    for (int e = T.pptr[t]; e < T.pptr[t + 1]; ++e) v += -s.P[T.plink[e] & 0x7fff];
    wp<FT>(s)[T.pslot[t]] = (FT)v;
  }
  for (int t = tid; t < n.nfill; t += NT) wp<FT>(s)[T.fill[t]] = FT(0);
  gsync<NT>();
}

// Coefficients at the current state for polish / terminal (autodiff.py:786-875):
// P, Y per link; emh per junction.
// With Pf / Ef (the P of every link and 1/hg of every emitter slot that the
// factor in use was formed with), `far` reports whether any of them moved
// by more than tol, relative; their loads are issued before the
// coefficients are formed.
template <int NT>
__device__ void adj_coeffs(const DevNet& n, const PumpTh& th, const Sh& s, const double* rrow,
                           const double* kerow, const double* Pf = nullptr,
                           const double* Ef = nullptr, double tol = 0.0,
                           bool* far = nullptr) {
  const int tid = gtid<NT>();
  bool fr = false;
  for (int k = tid; k < n.L; k += NT) {
    const double p0 = Pf ? Pf[k] : 0.0;
    double P, Y;
    link_coef(n, th, k, s.q[k], s.S[k], rrow[k], true, P, Y);
    s.P[k] = P;
    s.Y[k] = Y;
    if (Pf) fr = fr || !(fabs(P - p0) <= tol * fabs(p0));
  }
  const int nem = s.flag[2];
  for (int es = tid; es < nem; es += NT) {
    const double e0 = Ef ? Ef[es] : 0.0;
    double hl, hg;
    emitter_hl(n, s.em_e[es], s.em_ke[es], hl, hg);
    const double emh = 1.0 / hg;
    s.em_emh[es] = emh;
    if (Ef) fr = fr || !(fabs(emh - e0) <= tol * fabs(e0));
  }
  if (far) *far = fr;
  gsync<NT>();
}

// Primal reduced Newton solve with ACTIVE control valves (the system of
// dgga/autodiff.py:965-1029): an ACTIVE valve fixes the head it holds
// (dH_jc = -r_valve) and frees its flow, which enters the balance rows as the
// column u = sgn (e_jc - e_jo) (sgn +1 for a PRV, jc = n2; -1 for a PSV,
// jc = n1).  With dH_jc known, the unknowns are the other heads and the valve
// flow in slot jc: M y = r', M = the factored A with column jc replaced by u
// (the transpose of the adjoint's row-replaced matrix), r' = rhs - A_red[:,jc]
// dH_jc.  Woodbury on the factor: A^{-1} u_a - e_jc (one solve per active
// valve, right-hand side e_jc - e_jo), C_ab = X_b[jc_a], and `outer`
// refinement steps against the true M (one on the last polish step)
// make the result independent of the unrefined inner solves.  Output: dH
// (with dH_jc = -r_valve) and the valve flow corrections dqv[p].  rhs: V0
// (kept).
template <int NT, class FT, class TB>
__device__ void primal_solve(const DevNet& n, const TB& T, const Sh& s, double* rp, double* dH,
                             double* res, double* sx, double* cols, const double* rprv,
                             bool any_act, int outer, bool cols_ready) {
  const double* rhs = s.V0;
  double* t = s.V2;
  const int tid = gtid<NT>();
  if (!any_act) {  // `outer` refinement steps (one on the last polish step)
    solve_refined<NT, FT>(n, T, s, rhs, -1, dH, t, outer);
    return;
  }
  const int p = n.npcv;
  double* C = s.small;             // p*p
  double* y = s.small + 4 * p * p; // p
  double* actf = y + 2 * p;        // p
  double* dqv = actf + p;          // p, output
  if (tid == 0)
    for (int i = 0; i < p; ++i) actf[i] = s.S[n.pcv_link[i]] == WDS_ACTIVE ? 1.0 : 0.0;
  for (int q = tid; q < n.Nj; q += NT) sx[q] = 0.0;
  gsync<NT>();
  if (tid == 0)
    for (int i = 0; i < p; ++i)
      if (actf[i] != 0.0) sx[n.pcv_jc[i]] = -rprv[i];
  gsync<NT>();
  // r' = rhs - A_red dH_fixed (A_red: the factored matrix without the valves' penalty)
  for (int q = tid; q < n.Nj; q += NT) {
    double acc = amul_node(n, T, s, q, sx);
    for (int c = n.cb_ptr[q]; c < n.cb_ptr[q + 1]; ++c)
      acc -= sx[q] * (s.S[n.pcv_link[n.cb_idx[c]]] == WDS_ACTIVE ? kCBIG : 0.0);
    rp[q] = rhs[q] - acc;
  }
  gsync<NT>();
  // the outer refinement below contracts the error of these unrefined solves
  solve_refined<NT, FT>(n, T, s, rp, -1, dH, t, 0);
  // the columns and C depend on the factor alone: a step that reuses the
  // previous step's factor reuses them too (cols_ready)
  for (int c = 0; c < (cols_ready ? 0 : p); ++c) {  // X_c = A^{-1} sgn_c (e_jc - e_jo); zero for inactive valves
    double* xc = cols + (size_t)c * n.Nj;
    if (actf[c] == 0.0) {
      for (int q = tid; q < n.Nj; q += NT) xc[q] = 0.0;
      gsync<NT>();
      continue;
    }
    for (int q = tid; q < n.Nj; q += NT) res[q] = 0.0;
    gsync<NT>();
    if (tid == 0) {
      res[n.pcv_jc[c]] = n.pcv_sgn[c];
      res[n.pcv_jo[c]] = -n.pcv_sgn[c];
    }
    gsync<NT>();
    solve_refined<NT, FT>(n, T, s, res, -1, xc, t, 0);
  }
  if (tid == 0 && !cols_ready)
    for (int a0 = 0; a0 < p; ++a0)
      for (int c = 0; c < p; ++c)
        C[a0 * p + c] = actf[a0] != 0.0 ? cols[(size_t)c * n.Nj + n.pcv_jc[a0]]
                                         : (a0 == c ? 1.0 : 0.0);
  gsync<NT>();
  // x <- x - sum_b z_b (X_b - e_jc_b),  z = C^{-1} (x[jc] act)
  auto wood = [&](double* x) {
    if (tid == 0) {
      double* Cc = C + p * p;  // working copy (the small buffer holds 4 p^2 for C)
      for (int i = 0; i < p * p; ++i) Cc[i] = C[i];
      for (int a0 = 0; a0 < p; ++a0) y[a0] = x[n.pcv_jc[a0]] * actf[a0];
      dense_solve(Cc, y, p);
    }
    gsync<NT>();
    for (int q = tid; q < n.Nj; q += NT) {
      double acc = 0.0;
      for (int c = 0; c < p; ++c) acc += cols[(size_t)c * n.Nj + q] * y[c];
      x[q] = x[q] - acc;
    }
    gsync<NT>();
    if (tid == 0)
      for (int c = 0; c < p; ++c) x[n.pcv_jc[c]] += y[c] * actf[c];
    gsync<NT>();
  };
  wood(dH);
  for (int it = 0; it < outer; ++it) {
    // res = r' - M y, M y = A y_z + sum_a u_a y_jc (y_z: y with the valve slots zero)
    for (int q = tid; q < n.Nj; q += NT) sx[q] = dH[q];
    gsync<NT>();
    if (tid == 0)
      for (int i = 0; i < p; ++i)
        if (actf[i] != 0.0) sx[n.pcv_jc[i]] = 0.0;
    gsync<NT>();
    for (int q = tid; q < n.Nj; q += NT) res[q] = rp[q] - amul_node(n, T, s, q, sx);
    gsync<NT>();
    if (tid == 0)
      for (int i = 0; i < p; ++i)
        if (actf[i] != 0.0) {
          const double v = n.pcv_sgn[i] * dH[n.pcv_jc[i]];
          res[n.pcv_jc[i]] -= v;
          res[n.pcv_jo[i]] += v;
        }
    gsync<NT>();
    solve_refined<NT, FT>(n, T, s, res, -1, sx, t, 0);
    wood(sx);
    for (int q = tid; q < n.Nj; q += NT) dH[q] = dH[q] + sx[q];
    gsync<NT>();
  }
  if (tid == 0)
    for (int i = 0; i < p; ++i) {
      dqv[i] = actf[i] != 0.0 ? dH[n.pcv_jc[i]] : 0.0;
      if (actf[i] != 0.0) dH[n.pcv_jc[i]] = -rprv[i];
    }
  gsync<NT>();
}

__device__ __forceinline__ size_t al16(size_t x) { return (x + 15) / 16 * 16; }

__device__ Sh carve(const DevNet& n, unsigned char* base) {
  Sh s;
  size_t o = 0;
  auto take = [&](size_t bytes) { unsigned char* p = base + o; o = al16(o + bytes); return p; };
  s.q = nullptr;  // link flows and Y live in the global workspace (set by the kernel)
  s.Y = nullptr;
  s.P = (double*)take(8ull * n.L);
  if (n.fp32) {
    s.Wf = (float*)take(4ull * n.nnzL);
    s.W = nullptr;
  } else {
    s.W = (double*)take(8ull * n.nnzL);
    s.Wf = nullptr;
  }
  s.V0 = (double*)take(8ull * n.Nj);
  s.V1 = (double*)take(8ull * n.Nj);
  s.V2 = (double*)take(8ull * n.Nj);
  s.em_e = (double*)take(8ull * n.emcap);
  s.em_ke = (double*)take(8ull * n.emcap);
  s.em_emh = (double*)take(8ull * n.emcap);
  s.hf = (double*)take(8ull * (n.Nf > 0 ? n.Nf : 1));
  s.xf = (double*)take(8ull * (n.nxf > 0 ? n.nxf : 1));
  s.red = (double*)take(8ull * 4 * 32);
  s.small = (double*)take(8ull * (4 * n.npcv * n.npcv + 5 * n.npcv + 8));
  s.eslot = (int16_t*)take(2ull * n.Nj);
  s.tb = (double*)take(8ull * 2 * (WDS_TOP_MAX + 1));
  s.Mg = nullptr;  // set by the kernel
  s.wcnt = (int*)take(4ull * 32);
  s.flag = (int*)take(16);      // [0] factor verdict, [1] error, [2] emitter count
  s.err = s.flag + 1;
  s.S = (int8_t*)take(n.L);
  return s;
}

size_t smem_bytes(const DevNet& n) {
  auto a16 = [](size_t x) { return (x + 15) / 16 * 16; };
  size_t o = 0;
  o += a16(8ull * n.L);
  o += a16((n.fp32 ? 4ull : 8ull) * n.nnzL);
  o += 3 * a16(8ull * n.Nj);
  o += 3 * a16(8ull * n.emcap);
  o += a16(8ull * (n.Nf > 0 ? n.Nf : 1));
  o += a16(8ull * (n.nxf > 0 ? n.nxf : 1));
  o += a16(8ull * 4 * 32);
  o += a16(8ull * (4 * n.npcv * n.npcv + 5 * n.npcv + 8));
  o += a16(2ull * n.Nj);
  o += a16(8ull * 2 * (WDS_TOP_MAX + 1));
  o += a16(4ull * 32);
  o += a16(16);
  o += a16(n.L);
  return o;
}

// Compact the scenario's emitters (junctions with a positive coefficient, as
// given by val[jnode[p]] > 0) into slots in increasing elimination order:
// eslot[p] = slot or -1, em_ke = coefficient, em_e = initial flow 1.0
// (hydraul.c initial EmitterFlow).  Returns false when they exceed emcap.
template <int NT>
__device__ bool build_emitters(const DevNet& n, const Sh& s, const double* val, int stride_node) {
  const int tid = gtid<NT>(), lane = threadIdx.x & 31, warp = tid >> 5;
  int total = 0;
  bool over = false;
  for (int base = 0; base < n.Nj; base += NT) {
    const int p = base + tid;
    double v = 0.0;
    if (p < n.Nj) v = val[stride_node ? n.jnode[p] : p];
    const bool em = p < n.Nj && v > 0.0;
    const unsigned mask = __ballot_sync(0xffffffffu, em);
    if (lane == 0) s.wcnt[warp] = __popc(mask);
    gsync<NT>();
    int off = total, sum = 0;
    for (int w = 0; w < NT / 32; ++w) {
      if (w < warp) off += s.wcnt[w];
      sum += s.wcnt[w];
    }
    const int slot = off + __popc(mask & ((1u << lane) - 1u));
    if (p < n.Nj) {
      if (em && slot < n.emcap) {
        s.eslot[p] = (int16_t)slot;
        s.em_ke[slot] = v;
        s.em_e[slot] = 1.0;
        s.em_emh[slot] = 0.0;
      } else {
        s.eslot[p] = -1;
        if (em) over = true;
      }
    }
    total += sum;
    gsync<NT>();
  }
  if (tid == 0) s.flag[2] = total < n.emcap ? total : n.emcap;
  if (tid == 0) *s.err = 0;
  return !gsync_or<NT>(over);
}

// ---------------------------------------------------------------- CTA scenario rounds
// The CTAs of a launch are persistent: CTA `blk` of the `nblk` that run a plan
// holds `groups` scenario groups of NT threads (groups beyond it, in a CTA
// with more threads, stay idle), and group g takes scenario
// b = (r * groups + g) * nblk + blk in rounds r = 0, 1, ... while b < B.  The
// first nblk scenarios of a round go to group 0 of every CTA, so a partial
// last round runs one group per SM instead of filling a few CTAs, and a group
// with fewer co-resident groups runs faster (the kernels are latency-bound).
// The schedule tables are staged into shared memory once per CTA; a group's
// scenario state is its own slice of shared memory (global memory, per
// scenario, on the large-network layout), reused from round to round behind a
// group barrier.  `one(T, s, b)` solves scenario b.
template <int NT, class TB, class One>
__device__ __forceinline__ void cta_rounds(const DevNet& n, const DevWork& w, int B,
                                           int state_bytes, int blk, int nblk, int groups,
                                           One&& one) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / NT;
  TB T;
  if constexpr (TB::kWide) {
    T = tab_view<TB>(n, (const unsigned char*)n.stab);
  } else {
    for (int i = threadIdx.x; i < n.stab_bytes / 16; i += blockDim.x)
      ((uint4*)smem_raw)[i] = n.stab[i];
    __syncthreads();
    T = tab_view<TB>(n, smem_raw);
  }
  if (g >= groups) return;  // a whole group; groups use their own barriers
  for (int r = 0;; ++r) {
    const long long bl = ((long long)r * groups + g) * nblk + blk;
    if (bl >= B) return;  // uniform per group
    const int b = (int)bl;
    if (r > 0) gsync<NT>();  // the previous scenario's last reads of the group state
    Sh s;
    if constexpr (TB::kWide)
      s = carve(n, w.state + (size_t)b * state_bytes);
    else
      s = carve(n, smem_raw + n.stab_bytes + (size_t)g * state_bytes);
    one(T, s, b);
  }
}

// ---------------------------------------------------------------- forward kernel
// Forward of scenario b by one scenario group.
template <int NT, class TB, class FT>
__device__ __forceinline__ void forward_one(const DevNet& n, const DevWork& w, const FwdArgs& a,
                                            const TB& T, Sh s, int b) {
  s.q = w.lk + (size_t)b * 2 * n.L;
  s.Y = s.q + n.L;
  s.Mg = w.M + (size_t)b * n.nT * n.nT;
  const double* rrow = a.r + (long long)b * a.r_stride;
  const double* kerow = a.ke + (long long)b * a.ke_stride;
  const double* drow = a.d + (long long)b * n.N;
  const double* rhrow = a.rh + (long long)b * n.N;
  const PumpTh th = pump_th(n, a, b);
  // the scenario's junction demands in elimination order, gathered once and
  // read coalesced by every assembly
  double* dj = w.dj + (size_t)b * n.Nj;
  for (int p = gtid<NT>(); p < n.Nj; p += NT) dj[p] = drow[n.jnode[p]];
  bool hf_nan = false;  // a reservoir/tank head that is NaN: nothing is solved
  for (int f = gtid<NT>(); f < n.Nf; f += NT) {
    const double h = rhrow[n.fnode[f]];
    hf_nan = hf_nan || isnan(h);
    s.hf[f] = h;
  }
  for (int k = gtid<NT>(); k < n.L; k += NT) {
    s.q[k] = a.q0 ? a.q0[(size_t)b * n.L + k] : n.q_init[k];
    s.S[k] = a.s0 ? a.s0[(size_t)b * n.L + k] : n.status0[k];
  }
  hf_nan = gsync_or<NT>(hf_nan);
  const bool em_ok = build_emitters<NT>(n, s, kerow, 1) && !hf_nan;
  if (a.e0) {  // warm start of the emitter flows (solver.py:2881-2887)
    for (int p = gtid<NT>(); p < n.Nj; p += NT) {
      const int es = s.eslot[p];
      if (es >= 0) s.em_e[es] = a.e0[(size_t)b * n.N + n.jnode[p]];
    }
    gsync<NT>();
  }
  const bool sm = a.sm != 0;
  const int maxtrials = sm ? a.max_iter + (n.extra_iter > 0 ? n.extra_iter : 0) : a.max_iter;
  int nextcheck = n.checkfreq;
  int iters = maxtrials + 1, info = WDS_INFO_UNCONVERGED;
  double relerr = 0.0;
  double dratio = 0.0;  // diag_ratio of the last iteration's assembled matrix
  const int rec_w = n.L + 2 * n.Nj;  // unrolled record: q [L], e [Nj], H [Nj] per iteration
  double* recb = a.rec ? a.rec + (size_t)b * maxtrials * rec_w : nullptr;
  for (int it = 1; it <= (em_ok ? maxtrials : 0); ++it) {
    if (recb) {  // state at the start of iteration it, for the unrolled reverse pass
      double* r = recb + (size_t)(it - 1) * rec_w;
      for (int k = gtid<NT>(); k < n.L; k += NT) r[k] = s.q[k];
      for (int p = gtid<NT>(); p < n.Nj; p += NT)
        r[n.L + p] = s.eslot[p] >= 0 ? s.em_e[s.eslot[p]] : 0.0;
    }
    // ---- headloss coefficients (the next link's flow and resistance, in L2,
    // are loaded while this link's coefficients are formed)
    {
      int k = gtid<NT>();
      double qn = k < n.L ? s.q[k] : 0.0, rn = k < n.L ? rrow[k] : 0.0;
      for (; k < n.L; k += NT) {
        const double qk = qn, rk = rn;
        const int kn = k + NT;
        if (kn < n.L) {
          qn = s.q[kn];
          rn = rrow[kn];
        }
        double P, Y;
        link_coef(n, th, k, qk, s.S[k], rk, false, P, Y);
        s.P[k] = P;
        s.Y[k] = Y;
      }
    }
    gsync<NT>();
    assemble_gga<NT, FT>(n, T, s, kerow, dj);
    if (a.diag && n.npcv > 0) {  // condition proxy (dgga/solver.py:3026-3032)
      double mx = 0.0, mn = kINF;
      for (int p = gtid<NT>(); p < n.Nj; p += NT) {
        const double dv = fabs((double)wp<FT>(s)[T.colptr[p]]);
        mx = fmax(mx, dv);
        mn = fmin(mn, dv);
      }
      block_maxmin<NT>(mx, mn, s.red);
      dratio = mx / fmax(mn, 1e-300);
    }
    if (!factor<NT, FT>(n, T, s)) {
      info = WDS_INFO_NOT_PD;
      iters = it;
      break;
    }
    // refinement only where it can matter for the convergence test (see
    // WdsForwardOpts.refine_band); relerr still holds the previous iteration's
    const bool refine_it = a.rband <= 0.0 || it > 20 || (it > 1 && relerr < a.rband);
    solve_refined<NT, FT>(n, T, s, s.V0, -1, s.V1, s.V2, refine_it ? a.refine : 0);
    if (recb) {
      double* r = recb + (size_t)(it - 1) * rec_w + n.L + n.Nj;
      for (int p = gtid<NT>(); p < n.Nj; p += NT) r[p] = s.V1[p];
    }
    // ---- newflows (hydsolver.c:358-514 as restated in solver.py:3092-3110)
    double sums[4] = {0.0, 0.0, 0.0, 0.0};
    {
      int k = gtid<NT>();
      double yn = k < n.L ? s.Y[k] : 0.0, qn = k < n.L ? s.q[k] : 0.0;  // next link's, from L2
      for (; k < n.L; k += NT) {
        const double yk = yn, qk = qn;
        const int kn = k + NT;
        if (kn < n.L) {
          yn = s.Y[kn];
          qn = s.q[kn];
        }
        const double dh = head_of(T.e1[k], s.V1, s.hf) - head_of(T.e2[k], s.V1, s.hf);
        double dq = yk - s.P[k] * dh;
        if ((n.flags[k] & WDS_F_CHP) && dq > qk) dq = qk / 2.0;
        const double q2 = qk - dq;
        s.q[k] = q2;
        sums[0] += fabs(dq);
        sums[1] += fabs(q2);
      }
    }
    for (int p = gtid<NT>(); p < n.Nj; p += NT) {
      const int es = s.eslot[p];
      if (es >= 0) {
        double hl, hg;
        emitter_hl(n, s.em_e[es], s.em_ke[es], hl, hg);
        const double dqe = (hl - (s.V1[p] - n.el[p])) / hg;
        const double en = s.em_e[es] - dqe;
        s.em_e[es] = en;
        sums[2] += fabs(dqe);
        sums[3] += fabs(en);
      }
    }
    block_sum<NT>(sums, 4, s.red);
    const double dqsum = sums[0] + sums[2], qsum = sums[1] + sums[3];
    relerr = qsum > a.hacc ? dqsum / qsum : dqsum;
    if (!sm) {
      if (!recb && !(relerr > a.hacc)) {  // the unrolled map runs all its iterations
        iters = it;
        info = 0;
        break;
      }
      continue;
    }
    // ---- batched status machine (hydsolve, solver.py:3126-3179)
    bool vchg = false;
    for (int i = gtid<NT>(); i < n.npcv; i += NT) {
      const int k = n.pcv_link[i];
      const double h1 = head_of(T.e1[k], s.V1, s.hf), h2 = head_of(T.e2[k], s.V1, s.hf);
      const double qk = s.q[k], hs = n.pcv_hset[i], ht = n.htol;
      const int sk = s.S[k];
      const double hml = n.pcv_km[i] * (qk * qk);
      const bool neg = qk < -n.qtol;
      int ns = sk;
      if (n.pcv_psv[i]) {  // psvstatus (hydstatus.c:302-359 as in dgga/solver.py:1736-1765)
        if (sk == WDS_ACTIVE)
          ns = neg ? WDS_CLOSED : (h2 + hml > hs + ht ? WDS_OPEN : WDS_ACTIVE);
        else if (sk == WDS_OPEN)
          ns = neg ? WDS_CLOSED : (h1 < hs - ht ? WDS_ACTIVE : WDS_OPEN);
        else if (sk == WDS_CLOSED)
          ns = (h2 > hs + ht && h1 > h2 + ht) ? WDS_OPEN
               : ((h1 >= hs + ht && h1 > h2 + ht) ? WDS_ACTIVE : WDS_CLOSED);
        else if (sk == WDS_XPRESSURE)
          ns = neg ? WDS_CLOSED : sk;
      } else if (sk == WDS_ACTIVE)
        ns = neg ? WDS_CLOSED : (h1 - hml < hs - ht ? WDS_OPEN : WDS_ACTIVE);
      else if (sk == WDS_OPEN)
        ns = neg ? WDS_CLOSED : (h2 >= hs + ht ? WDS_ACTIVE : WDS_OPEN);
      else if (sk == WDS_CLOSED)
        ns = (h1 >= hs + ht && h2 < hs - ht) ? WDS_ACTIVE
             : ((h1 < hs - ht && h1 > h2 + ht) ? WDS_OPEN : WDS_CLOSED);
      else if (sk == WDS_XPRESSURE)
        ns = neg ? WDS_CLOSED : sk;
      if (ns != sk) {
        vchg = true;
        if (a.schg)  // schedule record: the valve pass changed link k
          atomicOr(&a.schg[((size_t)b * maxtrials + (it - 1)) * ((n.L + 31) >> 5) + (k >> 5)],
                   1u << (k & 31));
      }
      s.S[k] = (int8_t)ns;
    }
    vchg = gsync_or<NT>(vchg);
    const bool conv = relerr <= a.hacc;
    const bool br_conv = conv && it <= a.max_iter;
    const bool br_per = !conv && it <= n.maxcheck && nextcheck == it;
    bool chg = false;
    if (br_conv || br_per) {
      for (int k = gtid<NT>(); k < n.L; k += NT) {
        const int st0 = s.S[k];
        int st = (st0 == WDS_XHEAD || st0 == WDS_TEMPCLOSED) ? WDS_OPEN : st0;
        const double dh = head_of(T.e1[k], s.V1, s.hf) - head_of(T.e2[k], s.V1, s.hf);
        const double qk = s.q[k];
        if (n.kind[k] == WDS_KIND_CVPIPE) {  // cvstatus
          const bool rev = qk < -n.qtol;
          if (fabs(dh) > n.htol)
            st = (dh < -n.htol || rev) ? WDS_CLOSED : WDS_OPEN;
          else if (rev)
            st = WDS_CLOSED;
        }
        if (th.own_sp()) {  // pumpstatus at the call's speed (dgga/solver.py:673-679)
          const double w = th.sp(k);
          if (n.kind[k] == WDS_KIND_PUMP && w > 0.0 && st >= WDS_OPEN) {
            const double hmax = (n.flags[k] & WDS_F_CHP) ? kBIG : w * w * n.phunit[k];
            st = (-dh > hmax + n.htol) ? WDS_XHEAD : WDS_OPEN;
          }
        } else if ((n.flags[k] & WDS_F_PUMP_LIVE) && st >= WDS_OPEN) {  // pumpstatus
          st = (-dh > n.phmax[k] + n.htol) ? WDS_XHEAD : WDS_OPEN;
        }
        if (n.kind[k] == WDS_KIND_FCV) {
          // fcvstatus (hydstatus.c:362-398 as in dgga/solver.py:1816-1826,
          // 1875-1877), from the status before the reopening
          st = st0;
          if (dh < -n.htol || qk < -n.qtol)
            st = WDS_XFCV;
          else if (st0 == WDS_XFCV && qk >= n.fcv_qs[n.link_fcv[k]])
            st = WDS_ACTIVE;
        }
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
        if (st != st0) {
          chg = true;
          if (a.schg)  // schedule record: link k changed in this check
            atomicOr(&a.schg[((size_t)b * maxtrials + (it - 1)) * ((n.L + 31) >> 5) + (k >> 5)],
                     1u << (k & 31));
        }
        s.S[k] = (int8_t)st;
      }
      chg = gsync_or<NT>(chg);
    }
    if (a.sflags && gtid<NT>() == 0)  // iteration it ran, and which link-status branch
      a.sflags[(size_t)b * maxtrials + (it - 1)] = 4 | (br_conv ? 1 : 0) | (br_per ? 2 : 0);
    const bool stat_change = br_conv && (chg || vchg);
    if (br_conv && stat_change) nextcheck = it + n.checkfreq;
    if (br_per) nextcheck += n.checkfreq;
    if (conv && (it > a.max_iter || !stat_change)) {
      iters = it;
      info = 0;
      break;
    }
  }
  if (recb && em_ok && info == WDS_INFO_UNCONVERGED) {  // K iterations done
    iters = maxtrials;
    info = 0;
  }
  gsync<NT>();
  // junction heads of the GGA solution stay in V1
  double* Hs = w.scr + (size_t)b * w.nscr * n.Nj;  // global copy of heads for the polish
  if (a.polish >= 0 && info == 0) {
    for (int p = gtid<NT>(); p < n.Nj; p += NT) Hs[p] = s.V1[p];
    gsync<NT>();
    double* rp = Hs + n.Nj;
    double* res = rp + n.Nj;
    double* sx = res + n.Nj;
    double* cols = sx + n.Nj;                          // 2p Woodbury columns
    // small buffer: C [4p^2], y [2p], actf [p], row1 [p], then r_prv [p]
    double* rprv = s.small + 4 * n.npcv * n.npcv + 4 * n.npcv;
    // Factor reuse: once the previous step moved the flows by at most
    // kReuseFlow, a step keeps the factor in use (and its Woodbury columns)
    // while every link conductance P and emitter term 1/hg of the step is
    // within kReuseStep, relative, of the values it was factored with (kept
    // in the workspace's P / emh rows until the terminal store).  The
    // Jacobian then differs from the factored one by at most that fraction
    // in every entry, so the step's correction differs from the Newton
    // correction by that fraction of itself, which in the quadratic regime
    // is below rounding; the last step's outer refinement runs against
    // the current operator.  The terminal state kept for the adjoint reuses
    // it within kReuseTerminal: every adjoint solve takes two refinement
    // steps against the terminal operator, which leave the cube of that
    // distance.
    double* Pf = w.P + (size_t)b * n.L;     // P of each link and 1/hg of each
    double* Ef = w.emh + (size_t)b * n.Nj;  // emitter slot of the factor in use
    bool have = false, reuse = false, settled = false;
    for (int step = 0; step <= a.polish; ++step) {
      bool far = false;
      const bool cand = have && settled;
      adj_coeffs<NT>(n, th, s, rrow, kerow, cand ? Pf : nullptr, cand ? Ef : nullptr,
                     step == a.polish ? kReuseTerminal : kReuseStep, &far);
      reuse = cand && !gsync_or<NT>(far);
      if (!reuse) {
        assemble_reduced<NT, FT>(n, T, s);
        if (!factor<NT, FT>(n, T, s)) {
          info = WDS_INFO_NOT_PD;
          break;
        }
        // each thread keeps the entries it compares (the same index mapping)
        for (int k = gtid<NT>(); k < n.L; k += NT) Pf[k] = s.P[k];
        for (int es = gtid<NT>(); es < s.flag[2]; es += NT) Ef[es] = s.em_emh[es];
        have = true;
      }
      if (step == a.polish) break;  // terminal factor: keep it
      // residuals (autodiff.py:1032-1050); r_l overwrites Y
      for (int k = gtid<NT>(); k < n.L; k += NT) {
        const double hl = s.P[k] != 0.0 ? s.Y[k] / s.P[k] : 0.0;
        s.Y[k] = hl - (head_of(T.e1[k], Hs, s.hf) - head_of(T.e2[k], Hs, s.hf));
      }
      bool any_act = false;
      for (int i = gtid<NT>(); i < n.npcv; i += NT) {
        const bool act = s.S[n.pcv_link[i]] == WDS_ACTIVE;
        rprv[i] = (Hs[n.pcv_jc[i]] - n.pcv_hset[i]) * (act ? 1.0 : 0.0);
        any_act |= act;
      }
      any_act = gsync_or<NT>(any_act);
      for (int p = gtid<NT>(); p < n.Nj; p += NT) {
        const int a0 = T.inc_ptr[p], m = T.inc_split[p], z = T.inc_ptr[p + 1];
        double mm = 0.0, bt = 0.0;
        for (int e = m; e < z; ++e) {
          const int k = inc_link(T, e);
          mm += s.q[k];
          bt += s.P[k] * s.Y[k];
        }
        for (int e = a0; e < m; ++e) {
          const int k = inc_link(T, e);
          mm += -s.q[k];
          bt += -(s.P[k] * s.Y[k]);
        }
        const int es = s.eslot[p];
        double re = 0.0, emh = 0.0;
        if (es >= 0) {
          double hl, hg;
          emitter_hl(n, s.em_e[es], s.em_ke[es], hl, hg);
          re = hl - (Hs[p] - n.el[p]);
          mm = mm - s.em_e[es];
          emh = s.em_emh[es];
        }
        mm = mm - dj[p];
        s.V0[p] = (mm - bt) + emh * re;
      }
      gsync<NT>();
      // a Newton step corrects the rounding of the step before it: only the
      // last polish step's solve sets the final state, so it alone refines
      primal_solve<NT, FT>(n, T, s, rp, s.V1, res, sx, cols, rprv, any_act,
                           step == a.polish - 1 ? 1 : 0, reuse);
      // dq, de, state update
      double mv[2] = {0.0, 0.0};  // sum |dq|, sum |q|
      for (int k = gtid<NT>(); k < n.L; k += NT) {
        const double b1 = junc_of(T.e1[k], s.V1), b2 = junc_of(T.e2[k], s.V1);
        double dq = -s.P[k] * (s.Y[k] + (b2 - b1));
        const int i = n.link_pcv[k];
        if (i >= 0 && s.S[k] == WDS_ACTIVE)  // the free valve flow, solved in slot jc
          dq = s.small[4 * n.npcv * n.npcv + 3 * n.npcv + i];
        const double q2 = s.q[k] + dq;
        s.q[k] = q2;
        mv[0] += fabs(dq);
        mv[1] += fabs(q2);
      }
      for (int p = gtid<NT>(); p < n.Nj; p += NT) {
        const int es = s.eslot[p];
        if (es >= 0) {
          double hl, hg;
          emitter_hl(n, s.em_e[es], s.em_ke[es], hl, hg);
          const double re = hl - (Hs[p] - n.el[p]);
          s.em_e[es] = s.em_e[es] + (-re + s.V1[p]) / hg;
        }
        Hs[p] = Hs[p] + s.V1[p];
      }
      block_sum<NT>(mv, 2, s.red);  // its barriers publish the updates above
      settled = mv[0] <= kReuseFlow * mv[1];
    }
    if (info == 0) {  // store the terminal state for the adjoint
      FT* Wt = reinterpret_cast<FT*>(w.W) + (size_t)b * n.nnzL;
      for (int t = gtid<NT>(); t < n.nnzL; t += NT) Wt[t] = wp<FT>(s)[t];
      for (int k = gtid<NT>(); k < n.L; k += NT) {
        const double q = s.q[k];
        w.P[(size_t)b * n.L + k] = s.P[k];
        double dr = 0.0;
        const int st = s.S[k];
        const bool closed = st <= WDS_CLOSED || zero_speed(n, th, k, n.kind[k]);
        if ((n.flags[k] & WDS_F_IS_PIPE) && !closed) {
          const double sgn = q < 0.0 ? -1.0 : 1.0, qa = q * sgn;
          const double hgr = n.hexp * rrow[k] * pow(fmax(qa, 1e-30), n.hexp - 1.0);
          if (hgr >= n.rqtol) dr = pow(qa, n.hexp) * sgn;
        }
        w.dr[(size_t)b * n.L + k] = dr;
        const int ip = n.link_pump[k];
        if (ip >= 0) {
          double* dp = w.dpump + (size_t)b * 3 * n.npump;
          pump_dtheta(n, th, k, q, st, dp[ip], dp[n.npump + ip], dp[2 * n.npump + ip]);
        }
      }
      for (int p = gtid<NT>(); p < n.Nj; p += NT) {
        const int es = s.eslot[p];
        double hge = 1.0, dke = 0.0, emh = 0.0;
        if (es >= 0) {
          const double ke = s.em_ke[es], ee = s.em_e[es];
          double hl;
          emitter_hl(n, ee, ke, hl, hge);
          const double ea = fabs(ee);
          const double pw = pow(fmax(ea, 1e-30), n.qexp - 1.0);
          const double raw = n.qexp * fmax(ke, kCSMALL) * pw;
          dke = (raw < n.rqtol || ke < kCSMALL) ? 0.0 : pw * ee;
          emh = s.em_emh[es];
        }
        w.emh[(size_t)b * n.Nj + p] = emh;
        w.hge[(size_t)b * n.Nj + p] = hge;
        w.dke[(size_t)b * n.Nj + p] = dke;
      }
      const int pc = n.npcv > 0 ? n.npcv : 1;
      for (int i = gtid<NT>(); i < n.npcv; i += NT)
        w.act[(size_t)b * pc + i] = s.S[n.pcv_link[i]] == WDS_ACTIVE ? 1 : 0;
    }
    for (int p = gtid<NT>(); p < n.Nj; p += NT) s.V1[p] = Hs[p];
    gsync<NT>();
  }
  gsync<NT>();
  if (hf_nan) info = WDS_INFO_BAD_HEAD;
  else if (!em_ok) info = WDS_INFO_EMITTER_CAP;
  if (gtid<NT>() == 0) w.valid[b] = (a.polish >= 0 && info == 0) ? 1 : 0;
  // ---- outputs
  double* hrow = a.head + (size_t)b * n.N;
  double* erow = a.emit + (size_t)b * n.N;
  for (int f = gtid<NT>(); f < n.Nf; f += NT) {
    hrow[n.fnode[f]] = s.hf[f];
    erow[n.fnode[f]] = 0.0;
  }
  for (int p = gtid<NT>(); p < n.Nj; p += NT) {
    const int nd = n.jnode[p];
    hrow[nd] = s.V1[p];
    const int es = s.eslot[p];
    erow[nd] = es >= 0 ? s.em_e[es] : 0.0;
  }
  for (int k = gtid<NT>(); k < n.L; k += NT) {
    a.flow[(size_t)b * n.L + k] = s.q[k];
    a.status[(size_t)b * n.L + k] = s.S[k];
  }
  if (gtid<NT>() == 0) {
    a.iters[b] = iters;
    a.relerr[b] = relerr;
    a.info[b] = info;
    if (a.diag) a.diag[b] = dratio;
  }
}

template <int NT, class TB, class FT>
__device__ __forceinline__ void forward_body(const DevNet& n, const DevWork& w, const FwdArgs& a,
                                             int state_bytes, int blk, int nblk, int groups) {
  cta_rounds<NT, TB>(n, w, a.B, state_bytes, blk, nblk, groups, [&](const TB& T, Sh s, int b) {
    forward_one<NT, TB, FT>(n, w, a, T, s, b);
  });
}

// ---------------------------------------------------------------- adjoint kernel
// Node adjoint with constraint rows (autodiff.py:1107-1154) and the
// theta contraction (autodiff.py:1246-1312).
// Adjoint of right-hand side b by one scenario group.
template <int NT, class TB, class FT>
__device__ __forceinline__ void adjoint_one(const DevNet& n, const DevWork& w, const AdjArgs& a,
                                            const TB& T, Sh s, int b) {
  // kept state of scenario bf (several right-hand sides per scenario read the
  // same factor); right-hand sides, results and scratch are per b
  const int bf = (a.v0 + b) / (a.rhs_per > 1 ? a.rhs_per : 1);
  s.Mg = w.M + (size_t)bf * n.nT * n.nT;  // terminal top-block inverse of the forward
  if (!w.valid[bf]) return;  // uniform per group
  const FT* Wt = reinterpret_cast<const FT*>(w.W) + (size_t)bf * n.nnzL;
  for (int t = gtid<NT>(); t < n.nnzL; t += NT) wp<FT>(s)[t] = Wt[t];
  for (int k = gtid<NT>(); k < n.L; k += NT) s.P[k] = w.P[(size_t)bf * n.L + k];
  const int pc = n.npcv > 0 ? n.npcv : 1;
  // status is only consulted for ACTIVE flags of PRVs
  for (int k = gtid<NT>(); k < n.L; k += NT) {
    const int i = n.link_pcv[k];
    s.S[k] = (i >= 0 && w.act[(size_t)bf * pc + i]) ? WDS_ACTIVE : WDS_OPEN;
  }
  gsync<NT>();
  // emitter slots from the stored 1/hgrad (positive exactly at emitters)
  build_emitters<NT>(n, s, w.emh + (size_t)bf * n.Nj, 0);
  for (int p = gtid<NT>(); p < n.Nj; p += NT) {
    const int es = s.eslot[p];
    if (es >= 0) s.em_emh[es] = w.emh[(size_t)bf * n.Nj + p];
  }
  gsync<NT>();
  const double* gH = a.gH + (size_t)b * n.N;
  const double* gQ = a.gQ + (size_t)b * n.L;
  const double* gE = a.gE + (size_t)b * n.N;
  // r = B^T P gQ - em gE / hge - gH
  for (int p = gtid<NT>(); p < n.Nj; p += NT) {
    const int a0 = T.inc_ptr[p], m = T.inc_split[p], z = T.inc_ptr[p + 1];
    double acc = 0.0;
    for (int e = m; e < z; ++e) {
      const int k = inc_link(T, e);
      acc += s.P[k] * gQ[k];
    }
    for (int e = a0; e < m; ++e) {
      const int k = inc_link(T, e);
      acc += -(s.P[k] * gQ[k]);
    }
    const int nd = n.jnode[p];
    const int es = s.eslot[p];
    s.V0[p] = (acc - (es >= 0 ? s.em_emh[es] : 0.0) * gE[nd]) - gH[nd];
  }
  bool any_act = false;
  for (int i = gtid<NT>(); i < n.npcv; i += NT) any_act |= s.S[n.pcv_link[i]] == WDS_ACTIVE;
  any_act = gsync_or<NT>(any_act);
  double* lam = s.V1;
  double* t = s.V2;
  if (!any_act) {
    solve_refined<NT, FT>(n, T, s, s.V0, -1, lam, t, 2);
  } else {
    const int p = n.npcv;
    double* scr = w.scr + (size_t)b * w.nscr * n.Nj;
    double* r2 = scr;
    double* res = r2 + n.Nj;
    double* sx = res + n.Nj;
    double* cols = sx + n.Nj;                 // p Woodbury columns
    double* C = s.small;
    double* y = C + p * p;
    double* actf = y + p;
    if (gtid<NT>() == 0)
      for (int i = 0; i < p; ++i) actf[i] = s.S[n.pcv_link[i]] == WDS_ACTIVE ? 1.0 : 0.0;
    for (int q = gtid<NT>(); q < n.Nj; q += NT) r2[q] = s.V0[q];
    gsync<NT>();
    if (gtid<NT>() == 0)
      for (int i = 0; i < p; ++i)
        // row jc: lam[n2] - lam[n1] = gQ of the free valve flow, i.e.
        // lam[jc] - lam[jo] = sgn gQ (PRV jc = n2, PSV jc = n1)
        if (actf[i] != 0.0) r2[n.pcv_jc[i]] = n.pcv_sgn[i] * gQ[n.pcv_link[i]];
    gsync<NT>();
    // unrefined solves: the two outer refinement steps below contract their error
    solve_refined<NT, FT>(n, T, s, r2, -1, lam, t, 0);
    for (int c = 0; c < p; ++c) {
      if (actf[c] == 0.0) {  // meets y = 0 in the correction
        for (int q = gtid<NT>(); q < n.Nj; q += NT) cols[(size_t)c * n.Nj + q] = 0.0;
        gsync<NT>();
        continue;
      }
      solve_refined<NT, FT>(n, T, s, nullptr, n.pcv_jc[c], cols + (size_t)c * n.Nj, t, 0);
    }
    if (gtid<NT>() == 0)
      for (int a0 = 0; a0 < p; ++a0)
        for (int c = 0; c < p; ++c) {
          const double cw = cols[(size_t)c * n.Nj + n.pcv_jc[a0]] - cols[(size_t)c * n.Nj + n.pcv_jo[a0]];
          C[a0 * p + c] = cw * actf[a0] * actf[c] + (a0 == c ? 1.0 - actf[a0] : 0.0);
        }
    gsync<NT>();
    auto wood = [&](double* x, const double* rr) {
      if (gtid<NT>() == 0) {
        double* Cc = actf + p;  // working copy, p^2 after C, y, actf in the small buffer
        for (int i = 0; i < p * p; ++i) Cc[i] = C[i];
        for (int a0 = 0; a0 < p; ++a0)
          y[a0] = (x[n.pcv_jc[a0]] - x[n.pcv_jo[a0]] - rr[n.pcv_jc[a0]]) * actf[a0];
        dense_solve(Cc, y, p);
      }
      gsync<NT>();
      for (int q = gtid<NT>(); q < n.Nj; q += NT) {
        double acc = 0.0;
        for (int c = 0; c < p; ++c) acc += cols[(size_t)c * n.Nj + q] * y[c];
        x[q] = x[q] - acc;
      }
      gsync<NT>();
    };
    wood(lam, r2);
    for (int it = 0; it < 2; ++it) {
      for (int q = gtid<NT>(); q < n.Nj; q += NT) res[q] = r2[q] - amul_node(n, T, s, q, lam);
      gsync<NT>();
      if (gtid<NT>() == 0)
        for (int i = 0; i < p; ++i)
          if (actf[i] != 0.0)
            res[n.pcv_jc[i]] = r2[n.pcv_jc[i]] - (lam[n.pcv_jc[i]] - lam[n.pcv_jo[i]]);
      gsync<NT>();
      solve_refined<NT, FT>(n, T, s, res, -1, sx, t, 0);
      wood(sx, res);
      for (int q = gtid<NT>(); q < n.Nj; q += NT) lam[q] = lam[q] + sx[q];
      gsync<NT>();
    }
  }
  // theta contraction
  double* gd = a.gd + (size_t)b * n.N;
  double* gke = a.gke + (size_t)b * n.N;
  double* grh = a.grh + (size_t)b * n.N;
  double* gr = a.gr + (size_t)b * n.L;
  const double* hge = w.hge + (size_t)bf * n.Nj;
  const double* dke = w.dke + (size_t)bf * n.Nj;
  for (int p = gtid<NT>(); p < n.Nj; p += NT) {
    const int nd = n.jnode[p];
    gd[nd] = lam[p];
    double g = 0.0;
    if (s.eslot[p] >= 0) {
      const double lam_e = (gE[nd] + lam[p]) / hge[p];
      g = -(lam_e * dke[p]);
    }
    gke[nd] = g;
    grh[nd] = 0.0;
  }
  const double* dr = w.dr + (size_t)bf * n.L;
  for (int k = gtid<NT>(); k < n.L; k += NT) {
    const double l1 = junc_of(T.e1[k], lam), l2 = junc_of(T.e2[k], lam);
    const double lam_l = s.P[k] * (gQ[k] - (l2 - l1));
    gr[k] = -(lam_l * dr[k]);
    if (a.gsp) {  // pump theta (dgga/autodiff.py:736-741): -lam_l d hloss / d theta
      const int ip = n.link_pump[k];
      double g0 = 0.0, g1 = 0.0, g2 = 0.0;
      if (ip >= 0) {
        const double* dp = w.dpump + (size_t)bf * 3 * n.npump;
        g0 = -(lam_l * dp[ip]);
        g1 = -(lam_l * dp[n.npump + ip]);
        g2 = -(lam_l * dp[2 * n.npump + ip]);
      }
      a.gsp[(size_t)b * n.L + k] = g0;
      a.gh0[(size_t)b * n.L + k] = g1;
      a.grp[(size_t)b * n.L + k] = g2;
    }
  }
  for (int f = gtid<NT>(); f < n.Nf; f += NT) {
    const int nd = n.fnode[f];
    double acc = 0.0;
    for (int e = n.finc_ptr[f]; e < n.finc_split[f]; ++e) {
      const int k = n.finc[e];
      const double l1 = junc_of(T.e1[k], lam), l2 = junc_of(T.e2[k], lam);
      acc += s.P[k] * (gQ[k] - (l2 - l1));
    }
    for (int e = n.finc_split[f]; e < n.finc_ptr[f + 1]; ++e) {
      const int k = n.finc[e];
      const double l1 = junc_of(T.e1[k], lam), l2 = junc_of(T.e2[k], lam);
      acc += -(s.P[k] * (gQ[k] - (l2 - l1)));
    }
    grh[nd] = acc + gH[nd];
    gd[nd] = 0.0;
    gke[nd] = 0.0;
  }
}

template <int NT, class TB, class FT>
__device__ __forceinline__ void adjoint_body(const DevNet& n, const DevWork& w, const AdjArgs& a,
                                             int state_bytes, int blk, int nblk, int groups) {
  cta_rounds<NT, TB>(n, w, a.B, state_bytes, blk, nblk, groups, [&](const TB& T, Sh s, int b) {
    adjoint_one<NT, TB, FT>(n, w, a, T, s, b);
  });
}

// ---------------------------------------------------------------- unrolled-K reverse
// dP/dq, dY/dq, dP/dr, dY/dr of one link on the branch its coefficients took
// (the formulas of solve_unrolled, dgga/autodiff.py:1495-1591, differentiated
// as autograd does: a clamped quantity is a constant, |q| is q sgn with sgn
// constant; a custom pump curve's segment is chosen from the detached flow).
__device__ void link_dcoef(const DevNet& n, int k, double q, int st, double r, double& Pq,
                           double& Yq, double& Pr, double& Yr) {
  Pq = Yq = Pr = Yr = 0.0;
  const int kd = n.kind[k];
  if (st <= WDS_CLOSED || (n.flags[k] & WDS_F_ZERO_SPEED)) {  // P = 1/CBIG, Y = q
    Yq = 1.0;
    return;
  }
  const double sgn = q < 0.0 ? -1.0 : 1.0, qa = q * sgn;
  double hg, hl, dhg, dhl;
  if (kd <= WDS_KIND_CVPIPE) {
    const double ex = n.hexp, qc = fmax(qa, 1e-30);
    const double hg0 = ex * r * pow(qc, ex - 1.0);
    const bool lin = hg0 < n.rqtol;
    hg = lin ? n.rqtol : hg0;
    hl = lin ? hg * qa : hg * qa / ex;
    dhg = (lin || !(qa > 1e-30)) ? 0.0 : ex * (ex - 1.0) * r * pow(qc, ex - 2.0);
    dhl = lin ? n.rqtol : dhg * qa / ex + hg / ex;
    const double dhg_r = lin ? 0.0 : ex * pow(qc, ex - 1.0);
    const double dhl_r = dhg_r * qa / ex;
    const double km = n.km[k];
    if (km > 0.0) {
      hl += km * qa * qa;
      dhl += 2.0 * km * qa;
      hg += 2.0 * km * qa;
      dhg += 2.0 * km;
    }
    Pq = -dhg * sgn / (hg * hg);
    Yq = (dhl * hg - hl * dhg) / (hg * hg);
    Pr = -dhg_r / (hg * hg);
    Yr = sgn * (dhl_r * hg - hl * dhg_r) / (hg * hg);
    return;
  }
  if (kd == WDS_KIND_TCV) {
    const double km = n.km_tcv[k];
    if (!(km > 0.0)) {
      Yq = 1.0;
      return;
    }
    const double hg0 = 2.0 * km * qa;
    const bool lin = hg0 < n.rqtol;
    hg = lin ? n.rqtol : hg0;
    dhg = lin ? 0.0 : 2.0 * km * sgn;
    hl = lin ? q * hg : q * hg / 2.0;
    dhl = lin ? hg : (hg + q * dhg) / 2.0;
    Pq = -dhg / (hg * hg);
    Yq = (dhl * hg - hl * dhg) / (hg * hg);
    return;
  }
  if (kd != WDS_KIND_PUMP) return;
  const int t = n.ptype[k];
  if (t == 3) {  // NOCURVE: P const, Y = q
    Yq = 1.0;
    return;
  }
  const double spc = fmax(n.pspeed[k], 1e-12);
  if (t == 2) {  // CUSTOM, segment frozen: hg const, hl = H0 w^2 + hg q
    Yq = 1.0;
    return;
  }
  const double pn = n.pn[k];
  const double h0e = spc * spc * n.ph0[k];
  const double re = n.pr[k] * pow(spc, 2.0 - pn);
  if (t == 0) {  // CONST_HP
    const double qa2 = fmax(qa * qa, 1e-30);
    const double raw = -re / qa2;
    const bool big = raw > kCBIG, sml = raw < n.rqtol;
    hg = big ? kCBIG : (sml ? n.rqtol : raw);
    dhg = (big || sml || !(qa * qa >= 1e-30)) ? 0.0 : 2.0 * re / (qa2 * qa2) * qa * sgn;
    const double qcc = sgn * fmax(qa, 1e-30);
    hl = (big || sml) ? -hg * q : re / qcc;
    dhl = (big || sml) ? -hg : (qa > 1e-30 ? -re / (qcc * qcc) : 0.0);
  } else if (pn == 1.0) {  // linear
    hg = re;
    dhg = 0.0;
    hl = h0e + re * q;
    dhl = re;
  } else {  // power function
    const double qc = fmax(qa, 1e-30);
    const double raw = pn * re * pow(qc, pn - 1.0);
    const bool sml = raw < n.rqtol;
    hg = sml ? n.rqtol : raw;
    dhg = (sml || !(qa > 1e-30)) ? 0.0 : pn * (pn - 1.0) * re * pow(qc, pn - 2.0) * sgn;
    const double nn = fmax(pn, 1e-30);
    hl = sml ? h0e + hg * q : h0e + hg * q / nn;
    dhl = sml ? hg : (dhg * q + hg) / nn;
  }
  Pq = -dhg / (hg * hg);
  Yq = (dhl * hg - hl * dhg) / (hg * hg);
}

// Derivatives of an emitter's hloss and hgrad in its flow e and its Ke.
__device__ __forceinline__ void emitter_dcoef(const DevNet& n, double e, double ke, double hge,
                                              double& hle_e, double& hge_e, double& hle_k,
                                              double& hge_k) {
  const double kea = fmax(ke, kCSMALL), dkea = ke > kCSMALL ? 1.0 : 0.0;
  const double ae = fabs(e), ea = fmax(ae, 1e-30);
  const double sg = e > 0.0 ? 1.0 : (e < 0.0 ? -1.0 : 0.0);
  const bool lin = n.qexp * kea * pow(ea, n.qexp - 1.0) < n.rqtol;
  hge_e = (lin || !(ae > 1e-30)) ? 0.0 : n.qexp * (n.qexp - 1.0) * kea * pow(ea, n.qexp - 2.0) * sg;
  hge_k = lin ? 0.0 : n.qexp * pow(ea, n.qexp - 1.0) * dkea;
  hle_e = lin ? n.rqtol : (hge_e * e + hge) / n.qexp;
  hle_k = lin ? 0.0 : hge_k * e / n.qexp;
}

// Reverse pass of the unrolled-K map (solve_unrolled's autograd,
// dgga/autodiff.py:1357-1664) for one scenario group.  From the record of the
// forward, iteration k's coefficients, node matrix and factor are rebuilt
// (the same functions as the forward), then:
//   q' = q - (Y - P dh): qb -> Yb, Pb, dh_b (or qb / 2 on the constant-HP half step)
//   e' = e - (hle - (H - el)) / hge: eb -> hle_b, hge_b, H_b
//   H = A^{-1} F:       Fb = A^{-1} H_b (A symmetric), Pb -= (Fb1 - Fb2)(H1 - H2)
//   F = Y terms + P H_fixed + emitter terms + Xflow(q, e, d)
// and the coefficients' derivatives carry Pb, Yb, hle_b, hge_b to the flows,
// emitter flows, resistances and Ke.  Node sums gather over the incidence
// lists (no atomics).  Scratch per scenario: qb [L], a link temporary [L],
// eb [Nj], Fb [Nj].
template <int NT, class TB, class FT>
__device__ __forceinline__ void unrolled_one(const DevNet& n, const DevWork& w, const UnrollArgs& u,
                                             const TB& T, Sh s, int b) {
  const int tid = gtid<NT>();
  s.q = w.lk + (size_t)b * 2 * n.L;
  s.Y = s.q + n.L;
  s.Mg = w.M + (size_t)b * n.nT * n.nT;
  const double* rrow = u.r + (long long)b * u.r_stride;
  const double* kerow = u.ke + (long long)b * u.ke_stride;
  const double* drow = u.d + (size_t)b * n.N;
  const double* rhrow = u.rh + (size_t)b * n.N;
  FwdArgs a0{};  // the network's own pump parameters
  const PumpTh th = pump_th(n, a0, b);
  double* dj = w.dj + (size_t)b * n.Nj;  // junction demands in elimination order
  for (int p = tid; p < n.Nj; p += NT) dj[p] = drow[n.jnode[p]];
  for (int f = tid; f < n.Nf; f += NT) s.hf[f] = rhrow[n.fnode[f]];
  for (int k = tid; k < n.L; k += NT) s.S[k] = u.s0 ? u.s0[(size_t)b * n.L + k] : n.status0[k];
  gsync<NT>();
  if (!build_emitters<NT>(n, s, kerow, 1)) return;  // uniform; the forward failed alike
  double* qb = u.scr + (size_t)b * (2 * n.L + 2 * n.Nj);
  double* tl = qb + n.L;
  double* eb = tl + n.L;
  double* Fb = eb + n.Nj;
  double* gd = u.gd + (size_t)b * n.N;
  double* grh = u.grh + (size_t)b * n.N;
  double* gke = u.gke + (size_t)b * n.N;
  double* gr = u.gr + (size_t)b * n.L;
  const double* gH = u.gH + (size_t)b * n.N;
  for (int i = tid; i < n.N; i += NT) {
    gd[i] = 0.0;
    grh[i] = 0.0;
    gke[i] = 0.0;
  }
  for (int k = tid; k < n.L; k += NT) {
    gr[k] = 0.0;
    qb[k] = u.gQ[(size_t)b * n.L + k];
  }
  for (int p = tid; p < n.Nj; p += NT)
    eb[p] = s.eslot[p] >= 0 ? u.gE[(size_t)b * n.N + n.jnode[p]] : 0.0;
  gsync<NT>();
  const int R = n.L + 2 * n.Nj;
  const double* recb = u.rec + (size_t)b * u.K * R;
  for (int kk = u.K - 1; kk >= 0; --kk) {
    const double* rr = recb + (size_t)kk * R;
    const bool last = kk == u.K - 1;
    for (int k = tid; k < n.L; k += NT) s.q[k] = rr[k];
    for (int p = tid; p < n.Nj; p += NT) {
      const int es = s.eslot[p];
      if (es >= 0) s.em_e[es] = rr[n.L + p];
      s.V1[p] = rr[n.L + n.Nj + p];
    }
    gsync<NT>();
    for (int k = tid; k < n.L; k += NT) {
      double P, Y;
      link_coef(n, th, k, s.q[k], s.S[k], rrow[k], false, P, Y);
      s.P[k] = P;
      s.Y[k] = Y;
    }
    gsync<NT>();
    assemble_gga<NT, FT>(n, T, s, kerow, dj);
    factor<NT, FT>(n, T, s);  // the forward factored this matrix: positive definite
    // (1) q' = q - dq: the head-difference adjoint of each link
    for (int k = tid; k < n.L; k += NT) {
      const double dh = head_of(T.e1[k], s.V1, s.hf) - head_of(T.e2[k], s.V1, s.hf);
      const double dq = s.Y[k] - s.P[k] * dh;
      const bool hit = (n.flags[k] & WDS_F_CHP) && dq > s.q[k];
      tl[k] = hit ? 0.0 : qb[k] * s.P[k];
    }
    gsync<NT>();
    // (2) H_b at the junctions (links, emitter update, output) -> V0; fixed heads -> grh
    for (int p = tid; p < n.Nj; p += NT) {
      double acc = 0.0;
      const int a = T.inc_ptr[p], m = T.inc_split[p], z = T.inc_ptr[p + 1];
      for (int e = a; e < m; ++e) acc += tl[inc_link(T, e)];
      for (int e = m; e < z; ++e) acc += -tl[inc_link(T, e)];
      if (last) acc += gH[n.jnode[p]];
      const int es = s.eslot[p];
      if (es >= 0) {
        double hle, hge;
        emitter_hl(n, s.em_e[es], s.em_ke[es], hle, hge);
        acc += eb[p] / hge;  // e' = e - (hle - (H - el)) / hge: de'/dH = 1/hge
      }
      s.V0[p] = acc;
    }
    for (int f = tid; f < n.Nf; f += NT) {
      double acc = 0.0;
      for (int e = n.finc_ptr[f]; e < n.finc_split[f]; ++e) acc += tl[n.finc[e]];
      for (int e = n.finc_split[f]; e < n.finc_ptr[f + 1]; ++e) acc += -tl[n.finc[e]];
      if (last) acc += gH[n.fnode[f]];
      grh[n.fnode[f]] += acc;
    }
    gsync<NT>();
    // (3) F_b = A^{-1} H_b
    solve_refined<NT, FT>(n, T, s, s.V0, -1, Fb, s.V2, 2);
    // (4) links: P_b, Y_b from q', A and F; carried to q and r
    for (int k = tid; k < n.L; k += NT) {
      const double q = s.q[k], P = s.P[k], Y = s.Y[k];
      const int c1 = T.e1[k], c2 = T.e2[k];
      const double dh = head_of(c1, s.V1, s.hf) - head_of(c2, s.V1, s.hf);
      const bool hit = (n.flags[k] & WDS_F_CHP) && (Y - P * dh) > q;
      const double dqb = -qb[k];
      const double uu = junc_of(c1, Fb) - junc_of(c2, Fb);
      const double vv = junc_of(c1, s.V1) - junc_of(c2, s.V1);
      double Pb = (hit ? 0.0 : -dqb * dh) - uu * vv;
      const double Yb = (hit ? 0.0 : dqb) + uu;
      double tg = 0.0;  // F = ... + P H_fixed at the junction end
      if (c1 < 0 && c2 >= 0) {
        Pb += Fb[c2] * s.hf[-c1 - 1];
        tg = Fb[c2] * P;
      } else if (c2 < 0 && c1 >= 0) {
        Pb += Fb[c1] * s.hf[-c2 - 1];
        tg = Fb[c1] * P;
      }
      tl[k] = tg;
      double Pq, Yq, Pr, Yr;
      link_dcoef(n, k, q, s.S[k], rrow[k], Pq, Yq, Pr, Yr);
      qb[k] = qb[k] + (hit ? dqb / 2.0 : 0.0) - uu + Pb * Pq + Yb * Yq;
      gr[k] += Pb * Pr + Yb * Yr;
    }
    gsync<NT>();
    // (5) fixed heads through the grounding terms; junctions: demand, emitters
    for (int f = tid; f < n.Nf; f += NT) {
      double acc = 0.0;
      for (int e = n.finc_ptr[f]; e < n.finc_ptr[f + 1]; ++e) acc += tl[n.finc[e]];
      grh[n.fnode[f]] += acc;
    }
    for (int p = tid; p < n.Nj; p += NT) {
      const double Fp = Fb[p];
      gd[n.jnode[p]] += -Fp;
      const int es = s.eslot[p];
      if (es < 0) continue;
      const double ee = s.em_e[es], ke = s.em_ke[es];
      double hle, hge, hle_e, hge_e, hle_k, hge_k;
      emitter_hl(n, ee, ke, hle, hge);
      emitter_dcoef(n, ee, ke, hge, hle_e, hge_e, hle_k, hge_k);
      const double dqe = (hle - (s.V1[p] - n.el[p])) / hge;
      const double dqeb = -eb[p];
      const double hleb = dqeb / hge + Fp / hge;
      const double hgeb = -dqeb * dqe / hge + Fp * s.V1[p] / (hge * hge) -
                          Fp * (hle + n.el[p]) / (hge * hge);
      eb[p] = eb[p] - Fp + hleb * hle_e + hgeb * hge_e;
      gke[n.jnode[p]] += hleb * hle_k + hgeb * hge_k;
    }
    gsync<NT>();
  }
}

template <int NT, class TB, class FT>
__device__ __forceinline__ void unrolled_body(const DevNet& n, const DevWork& w, const UnrollArgs& u,
                                              int state_bytes, int blk, int nblk, int groups) {
  cta_rounds<NT, TB>(n, w, u.B, state_bytes, blk, nblk, groups, [&](const TB& T, Sh s, int b) {
    unrolled_one<NT, TB, FT>(n, w, u, T, s, b);
  });
}

template <int NT, int GR, class TB, class FT>
__global__ void __launch_bounds__(NT * GR, 1) k_unrolled(DevNet n, DevWork w, UnrollArgs u,
                                                         int state_bytes) {
  unrolled_body<NT, TB, FT>(n, w, u, state_bytes, blockIdx.x, gridDim.x, GR);
}

template <int NT, int GR, class TB, class FT>
__global__ void __launch_bounds__(NT * GR, 1) k_forward(DevNet n, DevWork w, FwdArgs a,
                                                        int state_bytes) {
  forward_body<NT, TB, FT>(n, w, a, state_bytes, blockIdx.x, gridDim.x, GR);
}

template <int NT, int GR, class TB, class FT>
__global__ void __launch_bounds__(NT * GR, 1) k_adjoint(DevNet n, DevWork w, AdjArgs a,
                                                        int state_bytes) {
  adjoint_body<NT, TB, FT>(n, w, a, state_bytes, blockIdx.x, gridDim.x, GR);
}

// Several plans (networks of different sizes) in one launch: CTAs
// [job.cta0, next job's cta0) run the job's plan, with 3 groups of 256
// threads each (a plan that fits fewer groups in shared memory leaves the
// others idle; large-network plans run 3 scenarios per CTA from global memory).
template <class FT>
__global__ void __launch_bounds__(768, 1) k_forward_multi(const __grid_constant__ FwdJobs jobs) {
  int p = 0;
  while (p + 1 < jobs.n && (int)blockIdx.x >= jobs.j[p + 1].cta0) ++p;
  const FwdJob& J = jobs.j[p];
  if (J.n.wide)
    forward_body<256, LTab, FT>(J.n, J.w, J.a, J.state_bytes, blockIdx.x - J.cta0,
                                (J.a.B + J.groups - 1) / J.groups, J.groups);
  else
    forward_body<256, STab, FT>(J.n, J.w, J.a, J.state_bytes, blockIdx.x - J.cta0,
                                (J.a.B + J.groups - 1) / J.groups, J.groups);
}

template <class FT>
__global__ void __launch_bounds__(768, 1) k_adjoint_multi(const __grid_constant__ AdjJobs jobs) {
  int p = 0;
  while (p + 1 < jobs.n && (int)blockIdx.x >= jobs.j[p + 1].cta0) ++p;
  const AdjJob& J = jobs.j[p];
  if (J.n.wide)
    adjoint_body<256, LTab, FT>(J.n, J.w, J.a, J.state_bytes, blockIdx.x - J.cta0,
                                (J.a.B + J.groups - 1) / J.groups, J.groups);
  else
    adjoint_body<256, STab, FT>(J.n, J.w, J.a, J.state_bytes, blockIdx.x - J.cta0,
                                (J.a.B + J.groups - 1) / J.groups, J.groups);
}

}  // namespace

// Kernel selectors, one definition per instance source and factor precision
// (declared in wds_internal.h): the host stub of the kernel for the plan's
// layout and scenario groups per CTA.
#ifndef WDS_FP32
#define WDS_FP32 0
#endif
#if WDS_FP32
using KFT = float;
#define WDS_KSEL(name) name##_f32
#else
using KFT = double;
#define WDS_KSEL(name) name##_f64
#endif

}  // namespace wds
