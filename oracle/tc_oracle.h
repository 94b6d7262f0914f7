/* CPU oracle for the FMM gravity evaluation -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C FP64 restatement of the reference's force evaluation
 * (get_force_and_potential, integrator.h:459-562 / taichi_with_jerks/integrator.h:308-432,
 * on the theta-MAC traversal traverse_eager.h:151-216 / taichi_with_jerks/traverse_eager.h:125-168).
 * It is used only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg,
 * as the checker.  The product (taichi_collisional_b200) never links or calls it.
 *
 * Pinned against the reference itself: oracle/ref_harness.cpp compiles the reference's
 * own headers (oracle/Makefile -> oracle/_ref/), and tests/golden/ holds outputs of that
 * build (tests/golden/make_golden.py).
 */
#ifndef TC_ORACLE_H
#define TC_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define TCO_VARIANT_TOP 0   /* top-level tree: mutual M2L, tiny-cell P2P, no jerks   */
#define TCO_VARIANT_JERKS 1 /* taichi_with_jerks: one-sided M2L with Mdot, P2P jerks  */

typedef struct {
  int p;              /* expansion order (EXPANSION)                                  */
  int ncrit;          /* max bodies per leaf                                          */
  int variant;        /* TCO_VARIANT_*                                                */
  int use_shift;      /* jerks root-centre shift (taichi_with_jerks/build_tree.h:253-268) */
  double theta;       /* opening angle, |d|^2 theta^2 > (Ri+Rj)^2                     */
  double shift_u[3];  /* the three drand48() draws used by the shift                  */
  int direct_below;   /* N < direct_below -> whole evaluation is a direct sum          */
} tco_params;

typedef struct {
  long long n_cells, n_leaves, n_m2l, n_p2p, n_p2p_inter;
  int max_level;
} tco_stats;

/* Full evaluation; outputs in the caller's original body order.  flags: bit0 sink,
 * bit1 source (NULL = every body is both).  vx/vy/vz and jx/jy/jz may be NULL for the
 * top variant.  Returns 0 on success. */
int tco_evaluate(const tco_params* prm, int n, const double* x, const double* y, const double* z,
                 const double* vx, const double* vy, const double* vz, const double* m,
                 const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                 double* jx, double* jy, double* jz, tco_stats* st);

/* The time-step pass of the top-level tree (get_force_and_potential(bodies, true) on the
 * theta path: traverse_eager.h:151-203 with get_steps, P2P of kernel_fast_lean.h:462-548):
 * no M2L; near-field pot/acc only; timestep[i] = sum over the body's P2P source cells of
 * 1/tau_min^4 (dt_param scales tau).  Always builds the tree (n < ncrit gives one leaf).
 * Returns -1 for the jerks tree, whose theta path has no time-step pass. */
int tco_evaluate_steps(const tco_params* prm, double dt_param, int n, const double* x, const double* y,
                       const double* z, const double* vx, const double* vy, const double* vz, const double* m,
                       const unsigned char* flags, double* ax, double* ay, double* az, double* pot,
                       double* timestep, tco_stats* st);

/* Tree of the last tco_evaluate call (reference cell order: depth-first, child blocks
 * allocated when the parent is split).  Arrays sized by tco_last_ncell()/n. */
int tco_last_ncell(void);
void tco_last_cells(int* begin, int* nbody, int* nchild, int* child, int* level,
                    double* X /*3*ncell*/, double* R, int* perm /*n: sorted -> original*/);
/* Multipoles / locals of the last evaluation (ncell*NTERM each; Md/Ld NULL-able). */
void tco_last_expansions(double* M, double* Md, double* L, double* Ld);
/* Interaction lists of the last evaluation as visited by the reference recursion:
 * kind 0 = M2L, 1 = P2P; pairs (target cell, source cell).  Returns count; pass NULL
 * to query the size. */
long long tco_last_list(int kind, int* tgt, int* src);

/* FP64 direct summation at nt targets over all sources (no softening; r=0 skipped). */
void tco_direct(int n, const double* x, const double* y, const double* z, const double* vx,
                const double* vy, const double* vz, const double* m, int nt, const int* targets,
                double* ax, double* ay, double* az, double* pot, double* jx, double* jy,
                double* jz);

/* Kernel-level pieces (single cells), for known-answer tests. */
void tco_init(int p);
void tco_make_gnm(const double* dX, double* re, double* im, int p);
void tco_swap_xz(double* v, int p);
void tco_p2m(int p, int nb, const double* x, const double* y, const double* z, const double* vx,
             const double* vy, const double* vz, const double* m, const double* C, double* M,
             double* Md);
void tco_m2m(int p, const double* Mc, const double* Mdc, const double* dX, double* Mp,
             double* Mdp);
void tco_m2l_rotate(int p, const double* M, const double* Md, const double* dX, double* L,
                    double* Ld);
void tco_m2l_direct(int p, const double* M, const double* dX, double* L);
void tco_l2l(int p, const double* Lp, const double* Ldp, const double* dX, double* Lc,
             double* Ldc);
void tco_l2p(int p, const double* L, const double* Ld, const double* dX, const double* v,
             double* out7 /* pot, ax, ay, az, jx, jy, jz (accumulated) */);
int tco_miniball(int np, const double* pts /*3*np*/, double* c, double* r2);

/* system_kinetic_energy, system_potential_energy, system_center_of_mass (integrator.h:887-925):
 * per-term FP64 expressions summed in order in long double, as the reference does (G = 1).
 * out[9] = kinetic, potential, mass, centre of mass (3), centre-of-mass velocity (3). */
void tco_system_diagnostics(int n, const double* m, const double* x, const double* y, const double* z,
                            const double* vx, const double* vy, const double* vz, const double* pot,
                            double* out);
/* drift with COMPSUM (integrator.h:42, :642-656) on one axis: a = s; e += dt v (fused);
 * s = a + e; e += a - s. */
void tco_drift_compsum(int n, double* s, double* e, const double* v, double dt);

#ifdef __cplusplus
}
#endif
#endif
