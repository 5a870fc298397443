// Internal layout shared by the host planner (wds_plan.cu) and the kernels
// (wds_device.cuh, instantiated by wds_k_*.cu).  Not part of the public ABI.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "wds_b200.h"

namespace wds {

constexpr double kCSMALL = 1e-6;   // hydcoeffs.c CSMALL, dgga/solver.py:34
constexpr double kCBIG = 1e8;      // dgga/solver.py:35
constexpr double kBIG = 1e10;
constexpr double kQZERO = 1e-6;
// Columns of the dense top block at most (16 x 16 threads x 3 x 3 entries each
// hold the block in registers while it is inverted).
constexpr int WDS_TOP_MAX = 48;

// Device tables of one network.  Junction vectors are indexed by their
// elimination index p (0..Nj-1); link ends are "end codes": p >= 0 for a
// junction, -(f+1) for the f-th fixed-head node.
struct DevNet {
  int N, L, Nj, Nf, nnzL, nlev, npcv, ntl, npairs, nfill, nxf, nftask, nfpair;
  // links [L]
  const int* e1;
  const int* e2;
  const int8_t* kind;
  const uint8_t* flags;
  const int8_t* status0;
  const int8_t* ptype;
  const double* km;
  const double* km_tcv;
  const double* q_init;
  const double* ph0;
  const double* pr;
  const double* pn;
  const double* pspeed;
  const double* phmax;
  const double* phunit;   // [L] shut-off head at unit speed (pumpstatus)
  const int* link_pump;   // [L] pump index or -1
  int npump;
  const int* cptr;        // [L+1]
  const double* cx;
  const double* cy;
  const int* link_tl;     // [L] tank-link index or -1
  const int* link_pcv;    // [L] pcv index or -1
  // junctions, elimination order [Nj]
  const int* jnode;       // node index
  const double* el;       // elevation
  const int* inc_ptr;     // [Nj+1]
  const int* inc_split;   // [Nj] first n2-side entry
  const int* inc;         // link index of each incidence entry
  const int* node_xf;     // [Nj] Xflow save slot or -1
  const int* cb_ptr;      // [Nj+1] pcv valves whose downstream node is p
  const int* cb_idx;
  // fixed nodes [Nf]
  const int* fnode;
  const int* finc_ptr;    // [Nf+1]
  const int* finc_split;  // [Nf]
  const int* finc;
  // off-diagonal entries of A
  const int* pair_ptr;    // [npairs+1]
  const int* pair_link;
  const int* pair_slot;   // [npairs]
  const int* fill_slot;   // [nfill]
  // symbolic structure of L (column-major, diagonal first)
  const int* colptr;      // [Nj+1]
  const int* rowidx;      // [nnzL]
  const int* levptr;      // [nlev+1]
  const int* levcol;      // [Nj]
  const int* ftask_ptr;   // [nlev+1]
  const int4* ftask;      // {slot, pair_begin, pair_end, is_diag}
  const int* fpair;       // [3*nfpair] {s1, s2, diag slot of k}
  const int4* fitem;      // [Nj] level order: {j, row entry begin, end, diag slot}
  const int4* bitem;      // [Nj] level order: {j, colptr[j], colptr[j+1], 0}
  const int2* rent;       // row entries {slot of L_jk, k}, level order
  // status-machine PRVs [npcv]
  const int* pcv_link;
  const int* pcv_j1;
  const int* pcv_j2;
  const int* pcv_off;     // slot of (j1,j2)
  const int* pcv_xf;      // Xflow slot of jc
  const double* pcv_hset;
  const double* pcv_km;
  // the head an ACTIVE valve holds: PRV at j2 (flow enters it, sgn +1), PSV
  // at j1 (flow leaves it, sgn -1); jo is the other end
  const int* pcv_jc;
  const int* pcv_jo;
  const double* pcv_sgn;
  const int* pcv_psv;     // 1 for a PSV (psvstatus), 0 for a PRV
  // status-machine FCVs [nfcv] (valve pass and fcvstatus; never constraint rows)
  int nfcv;
  const int* link_fcv;    // [L] fcv index or -1
  const int* fcv_link;
  const int* fcv_j1;
  const int* fcv_j2;
  const int* fcv_off;     // factor slot of the (j1, j2) entry
  const int* fcv_xf1;     // Xflow slots of its ends read by later PRVs, or -1
  const int* fcv_xf2;
  const double* fcv_qs;   // flow setting (cfs)
  const double* fcv_km;
  // valve pass order [npcv + nfcv]: link order; v >= 0 PRV v, v < 0 FCV -1 - v
  const int* vord;
  // tank links [ntl]
  const int* tl_link;
  const int* tl_tank;     // fixed index
  const int* tl_other;    // end code
  const double* tl_qsign;
  const double* tl_hmax;
  const double* tl_hmin;
  const uint8_t* tl_flags;
  double hexp, qexp, rqtol, htol, qtol, ucf_flow, ucf_head;
  int checkfreq, maxcheck, extra_iter;
  // compact 16-bit copy of the hot schedule tables, staged into shared memory
  // once per CTA (see STabOff)
  const uint4* stab;
  int stab_bytes;
  int o_spair, o_fpair, o_colptr, o_rowidx, o_levptr, o_rptr, o_rent, o_mode, o_inc_ptr, o_inc_split, o_inc, o_e1, o_e2, o_pptr, o_plink, o_pslot, o_fill, o_dslot;
  // dense top block: levels [L0, nlev) = columns [cT, Nj), nT = Nj - cT
  // (nT = 0 and L0 = nlev when the network has none)
  int L0, cT, nT;
  // large network: slot-valued tables are 32-bit and stay in global memory
  // with the scenario state (one 256-thread CTA per scenario); otherwise the
  // 16-bit tables are staged into shared memory
  int wide;
  // factor and substitutions in FP32 (residuals, refinement and the Newton
  // update stay in FP64)
  int fp32;
  int emcap;  // emitters per scenario held in shared memory
};

// Workspace kept between the forward (implicit mode) and the adjoint.
struct DevWork {
  double* W;      // [B][nnzL] terminal factor (unscaled columns, 1/D on diagonal); float when fp32
  double* P;      // [B][L]
  double* dr;     // [B][L]
  double* emh;    // [B][Nj]
  double* hge;    // [B][Nj]
  double* dke;    // [B][Nj]
  int8_t* act;    // [B][max(npcv,1)]
  double* scr;    // [B][nscr][Nj] scratch vectors
  double* lk;     // [B][2][L] link flows q and Y of the forward
  double* M;      // [B][nT][nT] inverse of the top block's Schur complement
  unsigned char* state;  // [B][state bytes] scenario state of large networks (else null)
  double* dpump;  // [B][3][npump] dhloss/d(speed, H0, R) of each pump at the terminal state
  double* dj;     // [B][Nj] the scenario's junction demands in elimination order
  int nscr;
  int* valid;     // [B] 1 when the terminal state is stored
};

struct FwdArgs {
  int B;
  double hacc;
  int max_iter, sm, refine, polish;
  double rband;  // refine a GGA solve only when the previous relerr < rband (0: always)
  long long ke_stride, r_stride;
  const double* d;
  const double* rh;
  const double* ke;
  const double* r;
  double* rec;       // unrolled record [B][K][L + 2 Nj] (q, e, H per iteration) or null
  const double* q0;  // [B][L] warm-start flows or null
  const double* e0;  // [B][N] warm-start emitter flows or null
  // pump parameters of the call ([L] rows, stride 0 or L; null: the network's)
  const double* th_sp;
  const double* th_h0;
  const double* th_r;
  long long th_stride;
  double* head;
  double* flow;
  double* emit;
  int8_t* status;
  int* iters;
  double* relerr;
  int* info;
  double* diag;           // [B] diag_ratio, or null
  uint8_t* sflags;        // [B][maxtrials] schedule branch flags, or null
  uint32_t* schg;         // [B][maxtrials][ceil(L/32)] schedule change bits, or null
  const int8_t* s0;       // [B][L] initial statuses, or null (the network's)
};

struct AdjArgs {
  int B;
  const double* gH;
  const double* gQ;
  const double* gE;
  double* gd;
  double* grh;
  double* gke;
  double* gr;
  // pump-parameter gradients [B][L] (null: not wanted)
  double* gsp = nullptr;
  double* gh0 = nullptr;
  double* grp = nullptr;
  // several right-hand sides per kept scenario: row b of this call (the
  // (v0 + b)-th right-hand side) uses the kept state of scenario
  // (v0 + b) / rhs_per; 0 or 1 means one right-hand side per scenario
  int rhs_per = 1;
  int v0 = 0;
};

// Host-side symbolic data kept in the plan (for inspection and tests).
struct HostSym {
  int Nj = 0;
  std::vector<int> perm, iperm, parent, level, colptr, rowidx;
};

// Kernels run `groups` independent scenario groups of 256 threads per CTA;
// shared memory = schedule tables + groups * per-scenario state.
// Reverse pass of the unrolled-K map (wds_unrolled_adjoint)
struct UnrollArgs {
  int B, K;
  const double* rec;    // [B][K][L + 2 Nj] from the unrolled forward
  const double* d;      // [B][N]
  const double* rh;     // [B][N]
  const double* ke;
  long long ke_stride;
  const double* r;
  long long r_stride;
  const double* gH;     // [B][N]
  const double* gQ;     // [B][L]
  const double* gE;     // [B][N]
  double* gd;           // [B][N]
  double* grh;          // [B][N]
  double* gke;          // [B][N]
  double* gr;           // [B][L]
  double* scr;          // [B][2 L + 2 Nj]
  const int8_t* s0;     // [B][L] frozen statuses of the forward, or null (the network's)
};
int launch_unrolled(const DevNet& n, const DevWork& w, const UnrollArgs& u, int groups,
                    void* stream, std::string* err);
int launch_forward(const DevNet& n, const DevWork& w, const FwdArgs& a, int groups,
                   void* stream, std::string* err);
int launch_adjoint(const DevNet& n, const DevWork& w, const AdjArgs& a, int groups,
                   void* stream, std::string* err);
size_t state_smem_bytes(const DevNet& n);

// One plan's share of a multi-plan launch.  `groups` is the number of
// scenario groups (256 threads each) per 768-thread CTA; state_bytes and cta0
// are filled by the launcher.
struct FwdJob {
  DevNet n;
  DevWork w;
  FwdArgs a;
  int groups, state_bytes, cta0;
};
struct AdjJob {
  DevNet n;
  DevWork w;
  AdjArgs a;
  int groups, state_bytes, cta0;
};
constexpr int WDS_MULTI_MAX = 8;  // plans per multi-plan launch
struct FwdJobs {
  FwdJob j[WDS_MULTI_MAX];
  int n;
};
struct AdjJobs {
  AdjJob j[WDS_MULTI_MAX];
  int n;
};
int launch_forward_multi(FwdJobs& jobs, void* stream, std::string* err);
int launch_adjoint_multi(AdjJobs& jobs, void* stream, std::string* err);

// Kernel instances (wds_k_*.cu, one source per kernel kind compiled once per
// factor precision): the host stub for a layout (wide: large network, one
// group) and a count of scenario groups per CTA.
const void* forward_kernel_f64(int wide, int groups);
const void* forward_kernel_f32(int wide, int groups);
const void* adjoint_kernel_f64(int wide, int groups);
const void* adjoint_kernel_f32(int wide, int groups);
const void* unrolled_kernel_f64(int wide, int groups);
const void* unrolled_kernel_f32(int wide, int groups);
const void* forward_multi_kernel_f64();
const void* forward_multi_kernel_f32();
const void* adjoint_multi_kernel_f64();
const void* adjoint_multi_kernel_f32();

}  // namespace wds
