/*
 * wds_b200.h -- C ABI of the B200 batched GGA solver and implicit adjoint.
 *
 * The library replaces the linear-solver hooks and the per-iteration body of
 * the reference's batched GGA route (dgga/solver.py:2922-3179,
 * `_cudss_forward` :2630, `_cudss_factor` :2683, `_cudss_adjoint` :2653) and
 * the GPU implicit adjoint (dgga/autodiff.py:1157-1312, `_kf_prepare` /
 * `_kf_solve` :898-925).  A binding from the reference calls these entry
 * points through ctypes with plain pointers.
 *
 * Units are EPANET internal units (ft, cfs).  All array arguments of
 * wds_forward / wds_adjoint are DEVICE pointers owned by the caller; the plan
 * owns its workspace (the terminal factor and coefficients kept for the
 * adjoint) and frees it in wds_free.  Every call is asynchronous on the given
 * CUDA stream (cudaStream_t passed as void*; NULL = legacy default stream).
 *
 * Return codes: 0 ok; negative values are errors (see WDS_E_*).  Per-scenario
 * numerical failures (non-positive pivot, non-convergence) are reported in the
 * `info` output array, never by trapping on the device.
 */
#ifndef WDS_B200_H
#define WDS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* element kinds after the host-side set-up (reference link types mapped by
 * GGASolver.__init__, dgga/solver.py:195-216, 745-832) */
enum {
  WDS_KIND_PIPE = 0,      /* PIPE (H-W or C-M)                       */
  WDS_KIND_CVPIPE = 1,    /* pipe with check valve                   */
  WDS_KIND_TCV = 2,       /* throttle control valve                  */
  WDS_KIND_PUMP = 3,      /* pump (curve kind in pump_type)          */
  WDS_KIND_PRV_FIXED = 4, /* PRV with MISSING setting: fixed open/closed valve */
  WDS_KIND_PRV = 5,       /* PRV with a setting: status-machine valve */
  WDS_KIND_FCV = 6,       /* FCV with a flow setting: valve pass + fcvstatus (both ends junctions) */
  WDS_KIND_PSV = 7        /* PSV with a setting: status-machine valve holding H[n1] (both ends junctions) */
};

/* status codes (EPANET StatusType, dgga/solver.py:1279-1281) */
enum {
  WDS_XHEAD = 0, WDS_TEMPCLOSED = 1, WDS_CLOSED = 2, WDS_OPEN = 3,
  WDS_ACTIVE = 4, WDS_XFLOW = 5, WDS_XFCV = 6, WDS_XPRESSURE = 7
};

/* per-link flag bits */
enum {
  WDS_F_ZERO_SPEED = 1,   /* pump with speed 0: always the closed branch   */
  WDS_F_PUMP_LIVE = 2,    /* pump with speed > 0: pumpstatus applies        */
  WDS_F_CHP = 4,          /* constant-horsepower pump: half-step guard      */
  WDS_F_IS_PIPE = 8       /* CVPIPE or PIPE: carries a roughness gradient   */
};

/* tank-link flag bits (tankstatus, dgga/solver.py:536-568) */
enum {
  WDS_TL_OVERFLOW = 1, WDS_TL_IS_PUMP = 2, WDS_TL_PUMP_IN = 4, WDS_TL_PUMP_OUT = 8
};

/* error codes */
enum {
  WDS_OK = 0,
  WDS_E_ARG = -1,         /* bad argument                                  */
  WDS_E_CUDA = -2,        /* CUDA runtime error                            */
  WDS_E_NOMEM = -3,       /* allocation failed                             */
  WDS_E_UNSUPPORTED = -4, /* network outside the supported element set     */
  WDS_E_STATE = -5        /* adjoint called without a forward in implicit mode */
};

/* per-scenario info bits written by wds_forward */
enum {
  WDS_INFO_NOT_PD = 1,      /* a pivot of the LDL^T factor was <= 0 or not finite */
  WDS_INFO_UNCONVERGED = 2, /* GGA loop ran out of trials                         */
  WDS_INFO_EMITTER_CAP = 4, /* more emitters than the plan's emitter capacity     */
  WDS_INFO_BAD_HEAD = 8     /* a reservoir/tank head was NaN; nothing was solved */
};

/* Static network description (host pointers; copied by wds_plan). */
typedef struct WdsNetwork {
  int32_t n_nodes;               /* N                                       */
  int32_t n_links;               /* L                                       */
  const int8_t* node_type;       /* [N] 0 junction, otherwise fixed head    */
  const double* elev;            /* [N] elevation (ft)                      */
  const int32_t* link_n1;        /* [L] start node                          */
  const int32_t* link_n2;        /* [L] end node                            */
  const int8_t* link_kind;       /* [L] WDS_KIND_*                          */
  const uint8_t* link_flags;     /* [L] WDS_F_* bits                        */
  const double* km;              /* [L] minor-loss coefficient (link->Km)   */
  const double* km_tcv;          /* [L] effective TCV coefficient           */
  const double* q_init;          /* [L] initial flow (cfs)                  */
  const int8_t* status0;         /* [L] initial status code                 */
  const int8_t* pump_type;       /* [L] -1, 0 CONST_HP, 1 POWER_FUNC, 2 CUSTOM, 3 NOCURVE */
  const double* pump_h0;         /* [L] */
  const double* pump_r;          /* [L] */
  const double* pump_n;          /* [L] exponent (snapped to 1 within TINY) */
  const double* pump_speed;      /* [L] relative speed (link setting)       */
  const double* pump_hmax;       /* [L] shut-off head used by pumpstatus    */
  const int32_t* curve_ptr;      /* [L+1] custom-curve point ranges         */
  const double* curve_x;         /* custom-curve flows (user units)         */
  const double* curve_y;         /* custom-curve heads (user units)         */
  const double* prv_hset;        /* [L] valve setting: El[n2] + setting (ft) for WDS_KIND_PRV,
                                    El[n1] + setting (ft) for WDS_KIND_PSV, the flow
                                    setting (cfs) for WDS_KIND_FCV               */
  int32_t n_tank_links;
  const int32_t* tl_link;        /* [T] link index                          */
  const int32_t* tl_tank;        /* [T] tank node                           */
  const int32_t* tl_other;       /* [T] the link's other node               */
  const double* tl_qsign;        /* [T] +1 / -1                             */
  const double* tl_hmax;         /* [T] */
  const double* tl_hmin;         /* [T] */
  const uint8_t* tl_flags;       /* [T] WDS_TL_* bits                       */
  double hexp, qexp, rqtol, htol, qtol, ucf_flow, ucf_head;
  int32_t checkfreq, maxcheck, extra_iter;
  const int32_t* perm;           /* [Nj] elimination order of junction rows, or NULL */
  int32_t emitter_capacity;      /* emitters per scenario kept on chip (0: 64) */
  int32_t layout;                /* WDS_LAYOUT_*: where the schedule tables and the
                                    per-scenario state live (no counterpart in the
                                    reference, which holds everything in torch tensors) */
  int32_t factor_fp32;           /* 1: LDL^T factor and substitutions in FP32, every
                                    solve refined against the FP64 operator (the
                                    precision choice dense_refine / cudss_refine leave
                                    open, dgga/solver.py:182, 384); 0: FP64 */
  const double* pump_hunit;      /* [L] pumpstatus shut-off head at unit speed (BIG for
                                    constant-HP pumps), used when a call passes its own
                                    pump speeds; NULL: pump_hmax / pump_speed^2 */
  /* Schedule choices the planner otherwise takes from its cost model (no
   * counterpart in the reference; set by the autotuner,
   * wdsgpu_b200/tune.py).  Each 0 means the planner's choice.  They change
   * the schedule, not the algorithm: results agree within rounding. */
  int32_t groups_per_cta;        /* scenario groups of 256 threads per CTA, 1-4 */
  int32_t top_max;               /* most columns of the dense top block (1-48), -1: none */
  double level_barrier_cost;     /* cost of a group barrier in the per-level mode model
                                    (in dependent rounds; 0: 0.5) */
} WdsNetwork;

/* WdsNetwork.layout */
#define WDS_LAYOUT_AUTO   0      /* shared memory when it fits, else global             */
#define WDS_LAYOUT_SHARED 1      /* 16-bit tables and state in shared memory, or fail   */
#define WDS_LAYOUT_GLOBAL 2      /* 32-bit tables and state in global memory, one CTA
                                    per scenario (large networks)                         */

/* Options of one forward call. */
typedef struct WdsForwardOpts {
  double accuracy;               /* hacc (relerr threshold)                  */
  int32_t max_iter;              /* trials                                   */
  int32_t status_machine;        /* 1: batched status machine                */
  int32_t refine;                /* refinement steps per linear solve (2); see refine_band */
  int32_t polish_steps;          /* reduced Newton polish steps; <0: plain solve only */
  int64_t ke_stride;             /* row stride of ke (0: one row for all)    */
  int64_t r_stride;              /* row stride of r  (0: one row for all)    */
  /* Warm start (the q0 / e0 keywords of GGASolver.solve, dgga/solver.py:
   * 2876-2887): device arrays or NULL for the defaults (q = initial flows,
   * emitter flow 1 where Ke > 0). */
  const double* q0;              /* [B,L] initial link flows, or NULL        */
  const double* e0;              /* [B,N] initial emitter flows (read at junctions with Ke > 0), or NULL */
  /* Pump parameters of this call (the speed / pump_h0 / pump_r of
   * implicit_solve, dgga/autodiff.py:1315-1342): rows of [L] values read at
   * pump links, one row for all scenarios (pump_stride 0) or one per
   * scenario (pump_stride L); NULL: the network's own. */
  const double* pump_speed;      /* relative speed (link setting)           */
  const double* pump_h0;         /* curve coefficient H0                    */
  const double* pump_r;          /* curve coefficient R                     */
  int64_t pump_stride;
  /* Which GGA iterations refine their solve (dense_refine / cudss_refine of
   * the reference refine every one, dgga/solver.py:3056, 2647).  0: every
   * iteration.  > 0: an iteration refines when the previous iteration's
   * relerr is below refine_band (or past iteration 20); the others take one
   * unrefined FP64 substitution.  While relerr is far above the rounding an
   * unrefined solve adds (about 1e-11 to 1e-9 relative), the Newton
   * iteration corrects that rounding by itself.  GGASolver passes 1e-5 at
   * accuracy >= 1e-8 (where that rounding is also far below the convergence
   * test) and 0 at tighter accuracies.  Polish and adjoint solves always
   * refine. */
  double refine_band;
  /* Unrolled-K mode (solve_unrolled, dgga/autodiff.py:1357-1664): a device
   * array [B][max_iter][L + 2 Nj] or NULL.  When set, the call runs exactly
   * max_iter GGA iterations with no convergence test (status_machine must be
   * 0 and polish_steps < 0, the statuses stay frozen: status0 or the
   * network's initial ones; q0 / e0 give the starting flows) and records
   * each iteration's starting flows, emitter flows (by junction) and
   * solved junction heads there, for wds_unrolled_adjoint. */
  double* unroll_record;
  /* Condition proxy of GGASolver.solve's result dict (`diag_ratio`,
   * dgga/solver.py:3026-3032, 3205-3207): a device array [B] or NULL; per
   * scenario max |A_jj| / max(min |A_jj|, 1e-300) of the node matrix
   * assembled in its last GGA iteration (PRV valve coefficients and the CBIG
   * diagonal of ACTIVE valves included).  Written for networks with
   * status-machine PRVs/PSVs, zero otherwise. */
  double* diag_ratio;
  /* Status-machine schedule (record_schedule, dgga/solver.py:2740-2745,
   * 3136-3160): device arrays, zero on entry, or NULL.  sched_flags uint8
   * [B][T] (T = max_iter + max(extra_iter, 0)): bit 2 when the scenario ran
   * iteration t + 1, bit 0 when that iteration ran the link-status check on
   * the converged branch, bit 1 on the periodic branch; sched_chg uint32
   * [B][T][ceil(L / 32)]: bit k of a row set when the iteration's valve
   * status pass (PRV/PSV links) or link-status check (the other links)
   * changed link k's status. */
  uint8_t* sched_flags;
  uint32_t* sched_chg;
  /* Initial link statuses (WDS_XHEAD .. WDS_XPRESSURE), a device array
   * int8 [B][L], or NULL for the network's status0: the status warm start
   * of an extended-period step, which EpsDriver.run carries from frame to
   * frame (run_gga(status0=S), dgga/eps.py:366-373).  With unroll_record,
   * the frozen statuses of solve_unrolled's `status` (pass the same array
   * to wds_unrolled_adjoint). */
  const int8_t* status0;
} WdsForwardOpts;

typedef struct WdsPlan WdsPlan;

/* Symbolic analysis (ordering, elimination tree, level schedule) and device
 * tables for one network; workspace for up to `max_batch` scenarios.
 * Replaces GGASolver.__init__'s index build (dgga/solver.py:283-369) and
 * symbolic.build_symbolic (dgga/symbolic.py:475-514). */
int wds_plan(const WdsNetwork* net, int32_t max_batch, WdsPlan** out);

/* Batched forward: GGA Newton loop with status machine, optional polish and
 * terminal factorisation kept for wds_adjoint.  Replaces GGASolver.solve
 * (dgga/solver.py:2703-3212) and ImplicitGGASolveGPU.forward's polish
 * (dgga/autodiff.py:1172-1243).
 *   demand, fixed_head: [B,N]; ke: [B or 1, N]; r: [B or 1, L]
 *   head [B,N], flow [B,L], emitter [B,N], status int8 [B,L],
 *   iters int32 [B], relerr [B], info int32 [B] (WDS_INFO_* bits). */
int wds_forward(WdsPlan* plan, int32_t batch, const WdsForwardOpts* opts,
                const double* demand, const double* fixed_head,
                const double* ke, const double* r,
                double* head, double* flow, double* emitter, int8_t* status,
                int32_t* iters, double* relerr, int32_t* info, void* stream);

/* Reduced implicit adjoint on the terminal factor of the last implicit
 * forward (zero new factorisations).  Replaces ImplicitGGASolveGPU.backward
 * (dgga/autodiff.py:1246-1312).  gH, gE: [B,N]; gQ: [B,L]; outputs
 * gd, grh, gke: [B,N]; gr: [B,L] (per scenario; batch sums are the caller's). */
int wds_adjoint(WdsPlan* plan, int32_t batch, const double* gH,
                const double* gQ, const double* gE, double* gd, double* grh,
                double* gke, double* gr, void* stream);

/* wds_adjoint plus the pump-parameter gradients [B,L] (zero off pump links):
 * gspeed = dLoss/d(relative speed), gh0 = dLoss/d(curve H0), grp =
 * dLoss/d(curve R), per scenario, at the speeds / coefficients the forward
 * was given in WdsForwardOpts (or the network's own).  Replaces the pump
 * theta of the CPU adjoint ImplicitGGASolve.backward
 * (dgga/autodiff.py:660-756, coefficients from _pump_coeffs_np :122-218),
 * which sums these rows over the batch for [L] parameters. */
int wds_adjoint_pumps(WdsPlan* plan, int32_t batch, const double* gH,
                      const double* gQ, const double* gE, double* gd, double* grh,
                      double* gke, double* gr, double* gspeed, double* gh0, double* grp,
                      void* stream);

/* Gradient of the unrolled-K map (solve_unrolled, dgga/autodiff.py:
 * 1357-1664, differentiated there by torch autograd): after a wds_forward
 * with opts.unroll_record = record and max_iter = K, the reverse pass over
 * the K iterations maps the output adjoints gH [B,N], gQ [B,L], gE [B,N] to
 * gd, grh, gke [B,N] and gr [B,L] (per scenario; a shared parameter takes
 * the batch sum).  demand / fixed_head / ke / r are the forward's inputs.
 * scratch: device array [B][2 L + 2 Nj]; status0: the frozen statuses the
 * forward ran with (its opts.status0, the `status` of solve_unrolled) or
 * NULL for the network's.  Networks with control valves
 * (PRV/PSV/FCV with a setting) are refused, as by the reference.  Rebuilds
 * each iteration's factor in the plan's workspace, so a kept implicit state
 * is gone afterwards. */
int wds_unrolled_adjoint(WdsPlan* plan, int32_t batch, int32_t K, const double* record,
                         const double* demand, const double* fixed_head, const double* ke,
                         int64_t ke_stride, const double* r, int64_t r_stride,
                         const double* gH, const double* gQ, const double* gE, double* gd,
                         double* grh, double* gke, double* gr, double* scratch,
                         const int8_t* status0, void* stream);

/* Statistics of the plan: [Nj, nnz_L, n_levels, n_pairs, smem_bytes,
 * n_pcv, nnz_A_lower, threads]. */
int wds_plan_stats(const WdsPlan* plan, int64_t* out8);

/* Generation of the plan's kept state: a counter that changes with every
 * call that rewrites the plan's workspace (wds_forward, wds_forward_multi,
 * wds_unrolled_adjoint).  A caller that differentiates later records it
 * after its implicit forward and checks it before wds_adjoint, so that a
 * forward run in between (which replaces the terminal factor) is an error
 * and never a silent gradient of the other call.  The reference keeps one
 * factor per autograd context (`ctx.kf`, dgga/autodiff.py:1203-1243); here a
 * caller with several pending backwards gives each its own plan. */
int wds_state_generation(const WdsPlan* plan, int64_t* gen);

/* Host copy of the symbolic structure: perm [Nj], colptr [Nj+1],
 * rowidx [nnz_L], parent [Nj], level [Nj] (any pointer may be NULL). */
int wds_plan_symbolic(const WdsPlan* plan, int32_t* perm, int32_t* colptr,
                      int32_t* rowidx, int32_t* parent, int32_t* level);

/* Several adjoints per kept scenario, on the terminal factors of the last
 * implicit wds_forward (no new factorisation): row b of this call is
 * right-hand side number first + b and uses the kept state of scenario
 * (first + b) / rhs_per.  Arrays as in wds_adjoint with `batch` rows;
 * batch <= the plan's max_batch (the rows' scratch), and every row must fall
 * on a kept scenario.  Replaces the multi-column solve of
 * sensitivity_matrix (dgga/sensitivity.py:59-145: one splu per frame, then
 * lu.solve(V, trans='T') over m sensor columns). */
int wds_adjoint_rhs(WdsPlan* plan, int32_t batch, int32_t rhs_per, int32_t first,
                    const double* gH, const double* gQ, const double* gE, double* gd,
                    double* grh, double* gke, double* gr, void* stream);

/* Device arrays of one plan in a multi-plan call (shapes as in wds_forward /
 * wds_adjoint). */
typedef struct WdsForwardIO {
  const double* demand;
  const double* fixed_head;
  const double* ke;
  const double* r;
  double* head;
  double* flow;
  double* emitter;
  int8_t* status;
  int32_t* iters;
  double* relerr;
  int32_t* info;
} WdsForwardIO;

typedef struct WdsAdjointIO {
  const double* gH;
  const double* gQ;
  const double* gE;
  double* gd;
  double* grh;
  double* gke;
  double* gr;
} WdsAdjointIO;

/* Networks of different sizes in one launch: `nplans` (at most 8) plans, each
 * with its own batch, options and arrays, run by one persistent kernel whose
 * CTAs are split among the plans (shared-memory or large-network layout per
 * plan).  Same per-plan results as wds_forward; no counterpart in the
 * reference, whose solver holds one network (dgga/solver.py:160). */
int wds_forward_multi(int32_t nplans, WdsPlan* const* plans, const int32_t* batch,
                      const WdsForwardOpts* opts, const WdsForwardIO* io, void* stream);

/* Adjoint of the last implicit wds_forward_multi (or wds_forward) of every
 * plan, in one launch; per plan as wds_adjoint. */
int wds_adjoint_multi(int32_t nplans, WdsPlan* const* plans, const int32_t* batch,
                      const WdsAdjointIO* io, void* stream);

/* Size of the fixed device array used by wds_forward_noalloc (64 MiB). */
#define WDS_NOALLOC_SCRATCH_BYTES (64u << 20)

/* Forward without allocation (no counterpart in the reference, which always
 * allocates through torch).  For callers that cannot call cudaMalloc when
 * they solve: a control loop that allocates everything at start-up because
 * an allocation can stall it, or a host whose device memory belongs to
 * another allocator.  Same arguments and results as wds_forward, but the
 * per-scenario workspace lives in one fixed WDS_NOALLOC_SCRATCH_BYTES device
 * array held by every GPU that loads the library until the process exits,
 * so the call never calls cudaMalloc or cudaFree.  A batch whose workspace
 * exceeds the array (about 340 scenarios of a 782-junction network) is
 * rejected with WDS_E_ARG.  The first call on a device loads the library's
 * device code there, which creates the array; make that first call before
 * any stream capture.  Calls share the array and it keeps the last call's
 * contents: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.  The call does not
 * prepare wds_adjoint. */
int wds_forward_noalloc(const WdsPlan* plan, int32_t batch, const WdsForwardOpts* opts,
                        const double* demand, const double* fixed_head,
                        const double* ke, const double* r,
                        double* head, double* flow, double* emitter, int8_t* status,
                        int32_t* iters, double* relerr, int32_t* info, void* stream);

/* Release the plan and its device memory. */
int wds_free(WdsPlan* plan);

/* Last error message of this thread (static storage). */
const char* wds_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* WDS_B200_H */
