/* taichi_b200 -- B200-native FMM gravity evaluation behind a C ABI.
 *
 * This library replaces the force evaluation of QirongZhu/taichi_collisional:
 *
 *   void get_force_and_potential(Bodies& bodies, bool get_steps);
 *     declared integrator.h:44, defined integrator.h:459-562 (top-level tree) and
 *     taichi_with_jerks/integrator.h:308-432 (jerks tree); called by kick_naive
 *     (integrator.h:245), kick_gradient (:353) and kick (:424), and in the jerks tree by
 *     taichi_with_jerks/integrator.h:163 and :273.
 *
 * It computes, for every sink body, the acceleration F (G = 1), the potential p in the
 * reference's positive convention (p = +sum m/r) and, for the jerks tree, the jerk J,
 * using the reference's adaptive octree FMM with the theta opening criterion
 * (traverse_eager.h:151-216; taichi_with_jerks/traverse_eager.h:125-168).
 *
 * Differences from the reference boundary (all deliberate):
 *   - structure-of-arrays pointers instead of the AoS Body vector (exafmm.h:22-45);
 *   - results are written in the caller's order, so the Body::index round trip
 *     (integrator.h:190-301) is not needed and the caller's arrays are never reordered;
 *   - every call returns a status code instead of calling exit() (exafmm.h:8-13).
 *
 * All entry points are thread-compatible per context (one context per host thread).
 */
#ifndef TAICHI_B200_H
#define TAICHI_B200_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

#define TC_PMAX 16

typedef enum {
  TC_OK = 0,
  TC_ERR_ARG = 1,        /* bad argument (n <= 0, p out of range, NULL pointer) */
  TC_ERR_CUDA = 2,       /* a CUDA runtime call failed; see tc_last_error_string */
  TC_ERR_CAPACITY = 3,   /* an interaction list overflowed; the context grows and retries */
  TC_ERR_NAN_INPUT = 4,  /* a position or mass is NaN/Inf */
  TC_ERR_DEPTH = 5,      /* more than ncrit bodies share a level-21 cell (kept as one leaf) */
  TC_ERR_UNSUPPORTED = 6, /* option not available in this build */
  TC_ERR_TIMEOUT = 7      /* a bounded device-side wait (tensor-core far field) gave up; outputs invalid */
} tc_status;

typedef enum { TC_VARIANT_TOP = 0, TC_VARIANT_JERKS = 1 } tc_variant;
/* TC_PREC_FP64: every stage FP64 (parity with the reference at 1e-12).
 * TC_PREC_MIXED: near field (P2P) in FP32 with compensated sums, far field FP64.
 * TC_PREC_MIXED_M2L: near field as MIXED, and the M2L in FP32 as well: for p <= 12 the swap
 *   and translation contractions run on the tensor cores (tcgen05, TF32 hi/lo split, FP32
 *   accumulation), the phase rotations in FP32 on the CUDA cores. */
typedef enum { TC_PREC_FP64 = 0, TC_PREC_MIXED = 1, TC_PREC_MIXED_M2L = 2 } tc_precision;
typedef enum { TC_MEM_HOST = 0, TC_MEM_DEVICE = 1 } tc_memory;

typedef struct {
  int p;              /* expansion order, 1..TC_PMAX (reference: EXPANSION, exafmm.h:52)    */
  int ncrit;          /* max bodies per leaf (reference: ncrit, exafmm.h:113)               */
  double theta;       /* opening angle: accept if |d|^2 theta^2 > (Ri+Rj)^2                 */
  int variant;        /* tc_variant: which reference tree the evaluation restates          */
  int precision;      /* tc_precision                                                       */
  int use_shift;      /* jerks tree root-centre shift (taichi_with_jerks/build_tree.h:253)  */
  double shift_u[3];  /* the three uniform draws the shift uses (drand48 in the reference)   */
  int direct_below;   /* N below this -> direct sum; -1 = reference rule (top: ncrit,
                         jerks: 8000; integrator.h:462, taichi_with_jerks/integrator.h:311) */
  int device;         /* CUDA device ordinal                                               */
  int selector;       /* far-field order per pair: 0 fixed p (the reference), 1 analytic error
                         estimate (the reference's MAC estimate, traverse_eager.h:82-96),
                         2 learned (MLP, after tc_train_selector).  With a selector on,
                         accepted pairs of a leaf target whose body counts multiply to at most
                         512 ((p+1)/13)^3 are summed directly instead of by an M2L          */
  double selector_tol;/* per-pair budget: the predicted |acc error| of a pair's M2L at most tol
                         times the least |a| among the target cell's bodies in the previous
                         evaluation of the same bodies (the first evaluation runs at fixed p) */
  int judge_n;        /* >0: after each evaluation, FP64 direct sums at judge_n seeded bodies;
                         with a selector, an RMS relative acceleration error above judge_tol
                         makes the call redo the far field at the fixed order p             */
  double judge_tol;
  unsigned long long judge_seed;
  double softening;   /* Plummer softening eps of the pair interactions (near field, direct sums,
                         tc_direct_sums): 1/r -> 1/sqrt(r^2 + eps^2); r = 0 pairs stay skipped.
                         0 = the reference's Newtonian kernel (it has no softening).  The far
                         field keeps the Newtonian multipoles, whose difference is O(eps^2/r^2)
                         at the far-field separations; the time-step pass and the error MAC's
                         pre-pass estimate stay Newtonian.  No counterpart in the reference.   */
} tc_params;

typedef struct {
  long long n_bodies, n_cells, n_leaves, n_m2l, n_p2p, n_p2p_inter;
  int max_level;
  double ms_total, ms_tree, ms_upward, ms_traverse, ms_m2l, ms_p2p, ms_downward;
  long long n_launches; /* kernels launched by the last tc_evaluate */
  long long flags;      /* diagnostic bits of the last evaluation (1 M2L, 2 P2P, 4 frontier capacity
                           retries; 8 depth limit; 16 an enclosing ball hit its iteration cap) */
  int n_classes;                /* distinct M2L orders the last evaluation's pairs got     */
  int class_order[16];          /* those orders, lowest first                              */
  long long class_pairs[16];    /* M2L pairs selected at each order (a batch of 32 pairs runs
                                   at the largest order among them)                        */
  double m2l_flop_fraction;     /* sum over pairs of (q+1)^3 / (p+1)^3, divided by pairs   */
  double judge_rms;             /* RMS relative acceleration error at the judge's bodies   */
  int judge_redo;               /* 1 if the judge rejected the selector's step             */
} tc_stats;

typedef struct tc_ctx tc_ctx;

/* Fill *prm with the reference defaults (p = 12, ncrit = 64, theta = 0.4, jerks tree). */
void tc_default_params(tc_params* prm);

/* Create a context on prm->device.  Replaces the globals P/NTERM/ncrit/theta
 * (exafmm.h:111-114) and initKernel() (kernel_fast_lean.h:122-160). */
tc_status tc_create(const tc_params* prm, tc_ctx** out);
tc_status tc_destroy(tc_ctx* ctx);

/* Run work on this CUDA stream (cudaStream_t passed as void*; NULL = legacy default). */
tc_status tc_set_stream(tc_ctx* ctx, void* stream);

/* Each tree's own traversal: the error-controlled MAC that get_force_and_potential uses
 * (horizontalPass(cells, cells, 1, get_steps)), preceded by the reference's low-order pre-pass
 * that estimates each body's acceleration (acc_old) for the cells' min_acc.
 *   top tree:   integrator.h:459-562; pre-pass integrator.h:476-493, kernel_fast_lean.h:1358-1647
 *               (acc_old = sum of scalar estimates); MAC horizontalPassHigh, traverse_eager.h:
 *               61-148 (both f1 and f2, pre-test |d| > Ra + Rb, small cells to P2P);
 *   jerks tree: taichi_with_jerks/integrator.h:308-432; pre-pass integrator.h:326-360,
 *               kernel_fast_lean.h:1446-1780 (acc_old = |F| of the order-2 FMM, its near field
 *               in FP32); MAC taichi_with_jerks/traverse_eager.h:59-122 (one-sided f2 only,
 *               pre-test 0.4 |d|^2 > (Ra + Rb)^2).
 * force_accuracy is the reference's global (top exafmm.h:95, default 2e-7; jerks
 * taichi_with_jerks/exafmm.h:99, default 2e-8).  With on != 0, tc_evaluate and
 * tc_evaluate_steps of this context build their lists with it instead of the theta MAC.  Not
 * captured by tc_set_graph.  As the reference's first call: acc_old starts at zero every
 * evaluation (the reference's global body array carries it from call to call). */
tc_status tc_set_error_mac(tc_ctx* ctx, int on, double force_accuracy);
/* The pre-pass's acc_old of the last evaluation with the error MAC, per body (caller order, host). */
tc_status tc_get_acc_old(tc_ctx* ctx, double* acc_old);

/* The whole evaluation as one CUDA graph (no counterpart in the reference, which has no
 * device).  With on != 0, tc_evaluate replays a captured graph
 * when the call matches the one it was captured for (same n, memory kind, every input/output
 * pointer and every tc_params field); any other call runs the normal path, returns its results
 * and then captures the graph for that call.  The captured sequence reads every count on the
 * device and sizes its launches by capacities 25 % over the planning call's tree and lists; an
 * overflow (reported in the status block the graph copies back) re-runs the call on the normal
 * path and re-plans.  Host buffers (TC_MEM_HOST) must be pinned to be captured; with pageable
 * host buffers, the time-step pass, the order selector or TC_PREC_MIXED_M2L the normal path
 * runs.  tc_graph_ready reports whether the next matching call will replay. */
tc_status tc_set_graph(tc_ctx* ctx, int on);
int tc_graph_ready(const tc_ctx* ctx);
/* Why the last capture was abandoned (stage and CUDA error), or "" when it succeeded. */
const char* tc_graph_note(const tc_ctx* ctx);

/* One force evaluation: the replacement of get_force_and_potential(bodies, false).
 *   x,y,z,m          positions and masses (required)
 *   vx,vy,vz         velocities (jerks tree; may be NULL for the top tree)
 *   flags            per body bit0 = sink (Body::issink), bit1 = source (Body::issource);
 *                    NULL = every body is both
 *   ax,ay,az,pot     outputs, caller order (overwritten, not accumulated)
 *   jx,jy,jz         jerk outputs (jerks tree; may be NULL)
 *   mem              TC_MEM_HOST or TC_MEM_DEVICE for ALL the pointers above
 * Synchronous with respect to the host when mem == TC_MEM_HOST. */
tc_status tc_evaluate(tc_ctx* ctx, int n, const double* x, const double* y, const double* z,
                      const double* vx, const double* vy, const double* vz, const double* m,
                      const unsigned char* flags, double* ax, double* ay, double* az,
                      double* pot, double* jx, double* jy, double* jz, int mem);

/* Statistics of the last evaluation (list sizes, per-phase device times). */
tc_status tc_get_stats(tc_ctx* ctx, tc_stats* st);

/* Inspection of the last evaluation (parity tests): cells in breadth-first order and the
 * interaction lists (kind 0 = M2L, 1 = P2P) as (target cell, source cell) pairs sorted by
 * target then source.  Host pointers; pass NULL to query sizes via tc_get_stats. */
tc_status tc_get_cells(tc_ctx* ctx, int* begin, int* nbody, int* nchild, int* child, int* level,
                       double* X /* 3 per cell */, double* R, int* perm /* n */);
tc_status tc_get_lists(tc_ctx* ctx, int kind, int* tgt, int* src);
tc_status tc_get_expansions(tc_ctx* ctx, double* M, double* Md, double* L, double* Ld);

/* ---- learned far-field order selector (selector = 2) ----------------------------------- */
typedef struct {
  int samples, iters, n_classes;
  int class_order[6];
  double train_loss, val_loss; /* mean squared error of predicted log10 errors            */
  double seconds;
} tc_train_report;

/* Train the selector's network on pairs from this input: one fixed-order evaluation builds
 * the tree and lists, `nsamples` M2L pairs are drawn (seeded), each is evaluated at every
 * order class against exact P2P, and the 3x32 MLP is fitted with Adam for `iters` steps on
 * the GPU.  The weights stay in the context (tc_get/set_selector_weights). */
tc_status tc_train_selector(tc_ctx* ctx, int n, const double* x, const double* y, const double* z,
                            const double* vx, const double* vy, const double* vz, const double* m,
                            int mem, int nsamples, int iters, unsigned long long seed,
                            tc_train_report* rep);
/* Change the selector mode and tolerance of an existing context (tc_params.selector/_tol). */
tc_status tc_set_selector(tc_ctx* ctx, int selector, double tol);
/* Training data of the last tc_train_selector (host copies): features [n x 8] and labels
 * [n x n_classes] (log10 relative errors).  Pass NULL to query *n. */
tc_status tc_get_selector_data(tc_ctx* ctx, float* feat, float* labels, int* n, int* n_classes);
/* Network parameters + standardisation (8 means, 8 inverse deviations, output offset):
 * `w` holds tc_selector_nparam() floats, `norm` 17 floats. */
int tc_selector_nparam(tc_ctx* ctx);
tc_status tc_get_selector_weights(tc_ctx* ctx, float* w, float* norm);
tc_status tc_set_selector_weights(tc_ctx* ctx, const float* w, const float* norm);
/* One evaluation of the training loss and its gradient on the current device (host arrays),
 * for checking the hand-written backward pass. */
tc_status tc_mlp_loss_grad(int ns, int n_out, const float* feat, const float* labels, const float* w,
                           const float* norm, float* grad, float* loss);
/* Predicted log10 errors [ns x n_out] of the network for given features (host arrays), by the
 * same tensor-core (TF32 operands, FP32 accumulation) inference the order selection runs. */
tc_status tc_mlp_predict(int ns, int n_out, const float* feat, const float* w, const float* norm, float* pred);

/* FP64 leapfrog update on device arrays (the integrator step around each evaluation):
 *   v += a * dt_kick;  x += v * dt_drift
 * Restates kick (integrator.h:378-457, v += a dt) and drift (integrator.h:642-670,
 * x += v dt) for a single shared time step; device pointers only, on the context's stream. */
tc_status tc_kick_drift(tc_ctx* ctx, int n, double* x, double* y, double* z, double* vx, double* vy,
                        double* vz, const double* ax, const double* ay, const double* az,
                        double dt_kick, double dt_drift);

/* Limit, in GPU clock cycles, of every bounded device-side wait of this context's kernels (the
 * tensor-core far field's waits for its products); cycles <= 0 restores the default (4e9, about
 * two seconds).  A wait that runs out stops the kernel's work, waits (with the default limit)
 * for the products already in flight, frees its tensor memory and makes the call return
 * TC_ERR_TIMEOUT; the context stays usable.  Meant for testing that path.  No counterpart in
 * the reference. */
tc_status tc_set_wait_limit(tc_ctx* ctx, long long cycles);

/* One shared-time-step leapfrog step (kick-drift-kick) around a force evaluation, on device
 * arrays: v += a dt/2; x += v dt; (a, pot, j) <- tc_evaluate(x, v, m); v += a dt/2.
 * a (ax, ay, az) holds the previous step's accelerations on entry (zero before the first step)
 * and the new ones on return; jx..jz may be NULL (jerks tree only).  The reference's kick
 * (integrator.h:378-457) and drift (integrator.h:642-670) for one shared step.  With
 * tc_set_graph on, the whole step -- both kicks, the evaluation and the judge -- is one CUDA
 * graph replay (captured on the first call, as tc_evaluate's graph; a step and a plain
 * evaluation never share a graph).  No counterpart in the reference, whose integrators are
 * host code.  Asynchronous on the context's stream. */
tc_status tc_step_leapfrog(tc_ctx* ctx, int n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                           const double* m, double* ax, double* ay, double* az, double* pot, double* jx, double* jy,
                           double* jz, double dt);

/* System diagnostics on device arrays (n bodies; pot in the positive convention p = +sum m/r
 * that tc_evaluate writes).  Replaces system_kinetic_energy (integrator.h:887-895),
 * system_potential_energy (:897-904) and system_center_of_mass (:906-925), G = 1:
 *   out[0] = sum m |v|^2 / 2,  out[1] = sum m pot / 2,  out[2] = sum m,
 *   out[3..5] = sum m x / sum m,  out[6..8] = sum m v / sum m    (out: 9 host doubles).
 * The reference sums in long double; these sums are double-double, independent of the launch
 * shape (bitwise reproducible).  Total energy as the reference prints it: out[0] - out[1].
 * Synchronises the context's stream. */
tc_status tc_system_diagnostics(tc_ctx* ctx, int n, const double* m, const double* x, const double* y,
                                const double* z, const double* vx, const double* vy, const double* vz,
                                const double* pot, double* out);

/* Compensated drift on device arrays, replacing drift (integrator.h:642-656) with COMPSUM
 * (integrator.h:42): per axis a = x; e += dt v; x = a + e; e += a - x, where e (ex, ey, ez) is
 * the caller's running position error (the reference's particle::pos_e), zero initially.
 * e += dt v is one fused multiply-add, as the reference compiles for an FMA-capable x86
 * target.  Device pointers, the context's stream. */
tc_status tc_drift_compensated(tc_ctx* ctx, int n, double* x, double* y, double* z, double* ex, double* ey,
                               double* ez, const double* vx, const double* vy, const double* vz, double dt);

/* One step dt of the reference's block-time-step integrator, device-resident:
 * do_evolve (integrator.h:873-890) with evolve_split_hold_dkd (integrator.h:834-871; the HOLD
 * build), its split by time step (integrator.h:591-640), kick_naive with time steps
 * (integrator.h:182-311: timestep = (sum 1/tau^4)^(-1/4) from tc_evaluate_steps with dt_param),
 * kick of sinks by sources (integrator.h:378-457, with sink / source flags through
 * tc_evaluate), kick_cpu for systems of at most 128 bodies (integrator.h:65-96, direct sums)
 * and the compensated drift (tc_drift_compensated).  The top-level tree only; its MAC is the
 * context's (tc_set_error_mac(ctx, 1, force_accuracy) for the reference's own).
 * All arrays are the caller's device arrays of n entries, permuted in place as the reference's
 * split swaps its particles (id[] follows the bodies; fill it with 0..n-1 to track them);
 * ex, ey, ez are the running position errors (the reference's pos_e, zero initially);
 * timestep and pot are outputs (the last values computed, as in the reference's particles).
 * st (may be NULL) receives counts of the step. */
typedef struct {
  int n_evaluations;  /* FMM evaluations (time-step passes and kicks)          */
  int n_direct;       /* direct kicks of small systems (kick_cpu)             */
  int n_splits;
  int max_level;      /* deepest level of the time-step hierarchy             */
  double simtime;     /* time advanced as the reference's diag->simtime is    */
} tc_evolve_stats;
/* The reference's split (integrator.h:591-640) as a permutation, without moving anything:
 * perm[k] = index (into timestep[]) of the body that the reference's two-pointer swaps leave at
 * position k; *nfast = fast.n (bodies with timestep < |dt| first; a single fast body counts as
 * none, as in the reference).  timestep and perm are device arrays; synchronises the stream. */
tc_status tc_split_order(tc_ctx* ctx, int n, const double* timestep, double dt, int* perm, int* nfast);
tc_status tc_evolve_hold_dkd(tc_ctx* ctx, int n, double* x, double* y, double* z, double* ex, double* ey,
                             double* ez, double* vx, double* vy, double* vz, double* m, double* timestep,
                             double* pot, int* id, double dt_param, double dt, tc_evolve_stats* st);
/* The same step with the reference's default scheme, the force-gradient integrator of its
 * GRADIENT / OUTPUTACC build: do_evolve with evolve_split_omelyan (integrator.h:720-812) --
 * kicks of dt / 6 around the recursion and the drifts, and in the middle kick_gradient
 * (integrator.h:313-376): 2 dt / 3 kicks with the forces evaluated at x + acc dt^2 / 24, acc
 * being the force of the last kick_naive, whose GRADIENT form gives every body the least time
 * step of its system (integrator.h:254-299).  Arguments and outputs as tc_evolve_hold_dkd;
 * acc is kept inside the context (3 n doubles more).  Where kick_gradient stores an
 * uninitialised array as the potential, the potential stays as the preceding kick set it. */
tc_status tc_evolve_omelyan(tc_ctx* ctx, int n, double* x, double* y, double* z, double* ex, double* ey,
                            double* ez, double* vx, double* vy, double* vz, double* m, double* timestep,
                            double* pot, int* id, double dt_param, double dt, tc_evolve_stats* st);

/* Hermite 4th-order step with one shared time step (Makino & Aarseth 1992), consuming the
 * accelerations and jerks of the jerks tree; no counterpart in the reference, whose jerks tree
 * has no integrator that uses them.  Device pointers, the context's stream:
 *   tc_hermite_predict: save[12 n] <- (x, v, a, j) at t; x, v <- their Taylor predictions at
 *     t + dt (x + v dt + a dt^2/2 + j dt^3/6, v + a dt + j dt^2/2)
 *   (the caller evaluates a1, j1 at the predicted x, v with tc_evaluate)
 *   tc_hermite_correct: v <- v0 + (a0 + a1) dt/2 + (j0 - j1) dt^2/12,
 *                       x <- x0 + (v0 + v) dt/2 + (a0 - a1) dt^2/12.
 * save is the caller's device buffer (12 n doubles); nothing is allocated. */
tc_status tc_hermite_predict(tc_ctx* ctx, int n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                             const double* ax, const double* ay, const double* az, const double* jx,
                             const double* jy, const double* jz, double* save, double dt);
tc_status tc_hermite_correct(tc_ctx* ctx, int n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                             const double* ax, const double* ay, const double* az, const double* jx,
                             const double* jy, const double* jz, const double* save, double dt);

/* Measured arithmetic throughput of this GPU in GFLOP/s (kind 0: FP64 FMA, 1: FP32 FMA),
 * used as the roofline denominator of the FP64 / FP32 kernels.  Returns < 0 on error. */
double tc_probe_peak(tc_ctx* ctx, int kind);

/* Direct-summation evaluation that allocates no device memory.  It has no counterpart in the
 * reference; it serves callers that cannot call cudaMalloc -- for example a host program
 * whose own allocator already owns the GPU memory it may use, or a time-stepping loop that
 * must not stall on the implicit device synchronisation cudaMalloc/cudaFree bring.
 *
 * Same arithmetic as tc_evaluate's direct branch (every sink against every source, FP64,
 * r = 0 skipped; the jerk when `jerk` is non-zero).  All pointers are device pointers;
 * vx/vy/vz are required when jerk != 0, flags may be NULL.  Work is queued on `stream`
 * (cudaStream_t as void*; NULL = legacy default) and the call returns without waiting.
 * Its working storage is one fixed static device array per GPU that loads the library
 * (held until the process exits), sized for TC_NOALLOC_MAX_N bodies; larger n returns
 * TC_ERR_CAPACITY without doing any work.  The first call on a device looks that array
 * up (cudaGetSymbolAddress) with the caller's current device, under a lock, and keeps the
 * address for the life of the process; make that first call before any stream capture, and
 * do not call this entry point again on a device after cudaDeviceReset there (the kept
 * address belongs to the reset context).  Every call reuses the same array, and every entry a
 * call reads is written earlier in that same call, so nothing has to be cleared between
 * calls; calls that overlap on the GPU (different streams, or another host thread) race on
 * the array.  The library's own code never uses this array: contexts keep their own storage. */
#define TC_NOALLOC_MAX_N 16384
tc_status tc_evaluate_direct_noalloc(int n, const double* x, const double* y, const double* z,
                                     const double* vx, const double* vy, const double* vz,
                                     const double* m, const unsigned char* flags, double* ax,
                                     double* ay, double* az, double* pot, double* jx, double* jy,
                                     double* jz, int jerk, void* stream);

const char* tc_status_string(tc_status s);
const char* tc_last_error_string(tc_ctx* ctx);
int tc_pmax(void);
/* 1 if expansion order p has compiled kernels in this build. */
int tc_order_supported(int p);
/* get_force_and_potential(bodies, true) of the top-level tree (integrator.h:459-562 with
 * get_steps; traverse_eager.h:151-203): the time-step pass.  As in the reference, no M2L is
 * done -- pot and acc are the near-field (P2P) parts only -- and every P2P pair adds the
 * pairwise criterion of kernel_fast_lean.h:462-548: timestep[i] = sum over the body's P2P
 * source cells of 1 / tau_min^4 (the reference's Body::timestep after the call; its
 * integrator takes 1 / sqrt(sqrt(timestep))).  dt_param is the reference's dt_param
 * (exafmm.h:109).  Velocities are required.  Always builds the tree.  Returns
 * TC_ERR_UNSUPPORTED for the jerks tree, whose theta path has no time-step pass
 * (taichi_with_jerks/traverse_eager.h:125-155 ignores get_steps); use tc_evaluate there. */
tc_status tc_evaluate_steps(tc_ctx* ctx, int n, const double* x, const double* y, const double* z, const double* vx,
                            const double* vy, const double* vz, const double* m, const unsigned char* flags,
                            double dt_param, double* ax, double* ay, double* az, double* pot, double* timestep,
                            int mem);
/* FP64 direct sums at nt target bodies (caller indices targets[k] in [0, n)) over all n bodies
 * (no softening; r = 0 skipped; sources are the bodies with flag bit 1, all if flags is NULL):
 * out[7k..7k+6] = pot, ax, ay, az, jx, jy, jz (jerk zero unless vx, vy, vz are given).
 * Inputs as in tc_evaluate (mem says where x..m and flags live; targets and out are host
 * arrays).  Uses the context's device and stream but none of its evaluation state.  A
 * validation helper for accuracy statements: the sums of the reference's direct()
 * (traverse_eager.h:349-360 over P2P, kernel_fast_lean.h:462), restricted to chosen targets. */
tc_status tc_direct_sums(tc_ctx* ctx, int n, const double* x, const double* y, const double* z, const double* vx,
                         const double* vy, const double* vz, const double* m, const unsigned char* flags, int nt,
                         const int* targets, double* out, int mem);
/* Constant matrices of the tensor-core far field (TC_PREC_MIXED_M2L, order q <= 12): the
 * swap and translation bins, TF32 hi parts then lo parts, 256 floats per 16 x 16 bin in the
 * kernel's shared-memory layout.  Writes at most cap floats into out (may be NULL) and
 * returns the full count, or -1 if q has no tensor-core plan.  A host-only diagnostic (no
 * device work), used to check the plan against the FP64 rotation M2L.  No counterpart in
 * the reference. */
int tc_tc_bins(int q, float* out, int cap);

#ifdef __cplusplus
}
#endif
#endif
