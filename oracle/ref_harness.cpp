// Harness around the reference's own headers -- TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/Makefile against the reference sources where they lie (no source is
// copied into this repository); the results land in oracle/_ref/.  It drives the
// reference's theta-MAC force evaluation exactly as get_force_and_potential does
// (integrator.h:459-562 / taichi_with_jerks/integrator.h:308-432) but with
// horizontalPass(cells, cells, 0, false) (traverse_eager.h:206-216), i.e.
//   buildTree -> upwardPass -> horizontalPass(theta) -> downwardPass
// and exposes the per-body outputs in the caller's order, the cells, and the interaction
// lists (recorded by re-walking the reference recursion, traverse_eager.h:151-203, on the
// reference's own cells).
#include <cmath>
#include <cstring>
#include <list>
#include <vector>
#include <omp.h>
#include <sys/time.h>

#include "exafmm.h"
#include "kernel_fast_lean.h"
#include "traverse_eager.h"

using namespace exafmm;

#ifdef TCR_JERKS
static const int kJerks = 1;
#else
static const int kJerks = 0;
#endif

static Cells g_cells;
static std::vector<int> g_list_t[2], g_list_s[2];
static int g_init = 0;
static int g_high = 0;  // last evaluation used the error-controlled MAC

static double now_s() {
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static void record(Cell* Ci, Cell* Cj) {
  // same decisions as horizontalPass (top: traverse_eager.h:151-203; jerks: :125-155)
  real_t d[3];
  for (int k = 0; k < 3; k++) d[k] = Ci->X[k] - Cj->X[k];
  real_t R2 = (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) * theta * theta;
  int ci = (int)(Ci - &g_cells[0]), cj = (int)(Cj - &g_cells[0]);
  if (R2 > (Ci->R + Cj->R) * (Ci->R + Cj->R)) {
    if (!kJerks && ((Ci->NBODY <= 2 && Cj->NBODY <= 8) || (Cj->NBODY <= 2 && Ci->NBODY <= 8))) {
      g_list_t[1].push_back(ci);
      g_list_s[1].push_back(cj);
    } else {
      g_list_t[0].push_back(ci);
      g_list_s[0].push_back(cj);
    }
  } else if (Ci->NCHILD == 0 && Cj->NCHILD == 0) {
    g_list_t[1].push_back(ci);
    g_list_s[1].push_back(cj);
  } else if (Cj->NCHILD == 0 || (Ci->R >= Cj->R && Ci->NCHILD != 0)) {
    for (Cell* c = Ci->CHILD; c != Ci->CHILD + Ci->NCHILD; c++) record(c, Cj);
  } else {
    for (Cell* c = Cj->CHILD; c != Cj->CHILD + Cj->NCHILD; c++) record(Ci, c);
  }
}

#ifndef TCR_JERKS
// same decisions as horizontalPassHigh (traverse_eager.h:61-148) on the reference's own cells
// (Pn, min_acc, R, X after its upwardPass), for recording the error-MAC lists
static void record_high(Cell* Ci, Cell* Cj) {
  real_t d[3];
  for (int k = 0; k < 3; k++) d[k] = Ci->X[k] - Cj->X[k];
  real_t R2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  real_t f1 = 10, f2 = 10;
  real_t Ra = Ci->R, Rb = Cj->R, Ra_p_Rb = Ra + Rb;
  if (R2 > Ra_p_Rb * Ra_p_Rb) {
    real_t R = sqrt(R2), Rp = R2, pa = 1, pb = 1, Eba = 0, Eab = 0;
    for (int k = 0; k <= P; k++) {
      real_t fac = combinator_coef[P][k];
      Eab += Ci->Pn[P - k] * pb * fac;
      Eba += Cj->Pn[P - k] * pa * fac;
      pa *= Ra;
      pb *= Rb;
      Rp *= R;
    }
    real_t fac = 8 * fmax(Ra, Rb) / Ra_p_Rb / Rp;
    Eab *= fac;
    f1 = Eab / (force_accuracy * Cj->min_acc);
    Eba *= fac;
    f2 = Eba / (force_accuracy * Ci->min_acc);
  }
  int ci = (int)(Ci - &g_cells[0]), cj = (int)(Cj - &g_cells[0]);
  if (f2 < 1 && f1 < 1) {
    int k = ((Ci->NBODY <= 2 && Cj->NBODY <= 8) || (Cj->NBODY <= 2 && Ci->NBODY <= 8)) ? 1 : 0;
    g_list_t[k].push_back(ci);
    g_list_s[k].push_back(cj);
  } else if (Ci->NCHILD == 0 && Cj->NCHILD == 0) {
    g_list_t[1].push_back(ci);
    g_list_s[1].push_back(cj);
  } else if (Cj->NCHILD == 0 || (Ci->R >= Cj->R && Ci->NCHILD != 0)) {
    for (Cell* c = Ci->CHILD; c != Ci->CHILD + Ci->NCHILD; c++) record_high(c, Cj);
  } else {
    for (Cell* c = Cj->CHILD; c != Cj->CHILD + Cj->NCHILD; c++) record_high(Ci, c);
  }
}
#else
// same decisions as the jerks tree's horizontalPassHigh (taichi_with_jerks/traverse_eager.h:
// 59-122) on the reference's own cells: the one-sided test f2 only, its pre-test
// |d|^2 0.4 > (Ra + Rb)^2, and no small-cell P2P rule
static void record_high(Cell* Ci, Cell* Cj) {
  real_t d[3];
  for (int k = 0; k < 3; k++) d[k] = Ci->X[k] - Cj->X[k];
  real_t R2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  real_t f2 = 10;
  real_t Ra = Ci->R, Rb = Cj->R, Ra_p_Rb = Ra + Rb;
  if (R2 * 0.4 > Ra_p_Rb * Ra_p_Rb) {
    real_t R = sqrt(R2), Rp = std::pow(R, -(P + 1)), pa = 1, Eba = 0;
    for (int k = 0; k <= P; k++) {
      real_t fac = combinator_coef[P][k];
      Eba += Cj->Pn[P - k] * pa * fac;
      pa *= Ra;
    }
    real_t fac = 8 * fmax(Ra, Rb) * Rp;
    Eba *= fac;
    f2 = Eba / (force_accuracy * Ci->min_acc);
  }
  int ci = (int)(Ci - &g_cells[0]), cj = (int)(Cj - &g_cells[0]);
  if (f2 < 1) {
    g_list_t[0].push_back(ci);
    g_list_s[0].push_back(cj);
  } else if (Ci->NCHILD == 0 && Cj->NCHILD == 0) {
    g_list_t[1].push_back(ci);
    g_list_s[1].push_back(cj);
  } else if (Cj->NCHILD == 0 || (Ci->R >= Cj->R && Ci->NCHILD != 0)) {
    for (Cell* c = Ci->CHILD; c != Ci->CHILD + Ci->NCHILD; c++) record_high(c, Cj);
  } else {
    for (Cell* c = Cj->CHILD; c != Cj->CHILD + Cj->NCHILD; c++) record_high(Ci, c);
  }
}
#endif

static int run(int n, const double* x, const double* y, const double* z, const double* vx, const double* vy,
               const double* vz, const double* m, const unsigned char* flags, double th, int nc, long seed,
               int nthreads, double* ax, double* ay, double* az, double* pot, double* jx, double* jy,
               double* jz, double* times, bool get_steps, double* timestep, bool high = false);

extern "C" {

int tcr_expansion(void) { return EXPANSION; }
int tcr_jerks(void) { return kJerks; }

// The three drand48() draws the jerks tree build consumes after srand48(seed)
// (taichi_with_jerks/build_tree.h:262-264).
void tcr_shift_uniforms(long seed, double* u) {
  srand48(seed);
  for (int d = 0; d < 3; d++) u[d] = drand48();
}

// One theta-MAC force evaluation.  flags: bit0 sink, bit1 source (NULL: both).
// times[4] = build, upward, horizontal, downward seconds.  Returns number of cells.
int tcr_evaluate(int n, const double* x, const double* y, const double* z, const double* vx,
                 const double* vy, const double* vz, const double* m, const unsigned char* flags,
                 double th, int nc, long seed, int nthreads, double* ax, double* ay, double* az,
                 double* pot, double* jx, double* jy, double* jz, double* times) {
  return run(n, x, y, z, vx, vy, vz, m, flags, th, nc, seed, nthreads, ax, ay, az, pot, jx, jy, jz, times,
             false, NULL);
}

// The same evaluation with get_steps = true (horizontalPass(cells, cells, 0, true)): the
// time-step pass of the top-level tree (no M2L; P2P with the pairwise criterion,
// kernel_fast_lean.h:462-548).  timestep[i] = the body's accumulated sum of 1/tau^4.
int tcr_evaluate_steps(int n, const double* x, const double* y, const double* z, const double* vx,
                       const double* vy, const double* vz, const double* m, const unsigned char* flags,
                       double th, int nc, double dtp, int nthreads, double* ax, double* ay, double* az,
                       double* pot, double* timestep) {
  dt_param = dtp;
  return run(n, x, y, z, vx, vy, vz, m, flags, th, nc, 1, nthreads, ax, ay, az, pot, NULL, NULL, NULL, NULL,
             true, timestep);
}

#ifndef TCR_JERKS
// The top tree's own get_force_and_potential (integrator.h:459-562): low-order pre-pass
// (acc_old), then the error-controlled MAC (horizontalPass(cells, cells, 1, get_steps)) with
// force_accuracy (exafmm.h:95, the global).  Same outputs as tcr_evaluate.
int tcr_evaluate_high(int n, const double* x, const double* y, const double* z, const double* vx,
                      const double* vy, const double* vz, const double* m, const unsigned char* flags,
                      double fa, int nc, int nthreads, double* ax, double* ay, double* az, double* pot) {
  force_accuracy = fa;
  return run(n, x, y, z, vx, vy, vz, m, flags, 0.4, nc, 0, nthreads, ax, ay, az, pot, nullptr, nullptr, nullptr,
             nullptr, false, nullptr, true);
}
// the same with get_steps = true (the time-step pass through the error-controlled MAC)
int tcr_evaluate_high_steps(int n, const double* x, const double* y, const double* z, const double* vx,
                            const double* vy, const double* vz, const double* m, const unsigned char* flags,
                            double fa, int nc, double dtp, int nthreads, double* ax, double* ay, double* az,
                            double* pot, double* timestep) {
  force_accuracy = fa;
  dt_param = dtp;
  return run(n, x, y, z, vx, vy, vz, m, flags, 0.4, nc, 0, nthreads, ax, ay, az, pot, nullptr, nullptr, nullptr,
             nullptr, true, timestep, true);
}
#else
// The jerks tree's own get_force_and_potential (taichi_with_jerks/integrator.h:308-432) without
// its direct-sum branch for small N: low-order pre-pass (acc_old = |F| of the order-2 FMM),
// then the error-controlled MAC (horizontalPass(cells, cells, 1, false)) with force_accuracy.
// seed feeds srand48 before buildTree (the root shift's draws).
int tcr_evaluate_high_jerks(int n, const double* x, const double* y, const double* z, const double* vx,
                            const double* vy, const double* vz, const double* m, const unsigned char* flags,
                            double fa, int nc, long seed, int nthreads, double* ax, double* ay, double* az,
                            double* pot, double* jx, double* jy, double* jz) {
  force_accuracy = fa;
  return run(n, x, y, z, vx, vy, vz, m, flags, 0.4, nc, seed, nthreads, ax, ay, az, pot, jx, jy, jz, nullptr,
             false, nullptr, true);
}
#endif
}  // extern "C"

static int run(int n, const double* x, const double* y, const double* z, const double* vx, const double* vy,
               const double* vz, const double* m, const unsigned char* flags, double th, int nc, long seed,
               int nthreads, double* ax, double* ay, double* az, double* pot, double* jx, double* jy,
               double* jz, double* times, bool get_steps, double* timestep, bool high) {
  if (!g_init) {
    P = EXPANSION;
    initKernel();
    g_init = 1;
  }
  theta = th;
  ncrit = nc;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  bodies.clear();
  bodies.resize(n);
  for (int i = 0; i < n; i++) {
    Body& b = bodies[i];
    b.X[0] = x[i]; b.X[1] = y[i]; b.X[2] = z[i];
    b.V[0] = vx ? vx[i] : 0; b.V[1] = vy ? vy[i] : 0; b.V[2] = vz ? vz[i] : 0;
    b.q = m[i];
    for (int d = 0; d < 3; d++) b.F[d] = 0;
#ifdef TCR_JERKS
    for (int d = 0; d < 3; d++) b.J[d] = 0;
#endif
    b.p = 0;
    b.acc_old = 0;
    b.timestep = 0;
    b.index = i;
    b.issink = flags ? (flags[i] & 1) : true;
    b.issource = flags ? ((flags[i] >> 1) & 1) : true;
  }
  srand48(seed);
  double t0 = now_s();
  g_cells = buildTree(bodies);
  double t1 = now_s();
  g_high = 0;
#ifndef TCR_JERKS
  if (high) {
    // integrator.h:476-539, in order
    g_high = 1;
    upwardPass_low(g_cells);
    horizontalPass_low(g_cells, g_cells);
    downwardPass_low(g_cells);
    for (size_t b = 0; b < bodies.size(); b++) {
      bodies[b].F[0] = bodies[b].F[1] = bodies[b].F[2] = 0;
      bodies[b].p = 0;
      bodies[b].timestep = 0;
    }
    for (size_t i = 0; i < g_cells.size(); i++)
      for (int term = 0; term < NTERM; term++) {
        g_cells[i].L[term] = 0;
        g_cells[i].M[term] = 0;
        g_cells[i].min_acc = HUGE;
        g_cells[i].has_sink = false;
      }
    upwardPass(g_cells);
    for (size_t i = 0; i < g_cells.size(); i++)
      for (int nn = 0; nn <= P; nn++) {
        for (int mm = -nn; mm <= nn; mm++) {
          int index = nn * nn + nn + mm;
          g_cells[i].Pn[nn] += g_cells[i].M[index] * g_cells[i].M[index] * factorial_table[nn + mm] *
                               factorial_table[nn - mm];
        }
        g_cells[i].Pn[nn] = sqrt(g_cells[i].Pn[nn]);
      }
  } else
#else
  if (high) {
    // taichi_with_jerks/integrator.h:326-398, in order
    g_high = 1;
    upwardPass_low(g_cells);
    horizontalPass_low(g_cells, g_cells);
    downwardPass_low(g_cells);
    for (size_t b = 0; b < bodies.size(); b++) {
      Body& B = bodies[b];
      B.acc_old = sqrt(B.F[0] * B.F[0] + B.F[1] * B.F[1] + B.F[2] * B.F[2]);
      B.F[0] = B.F[1] = B.F[2] = 0;
      B.J[0] = B.J[1] = B.J[2] = 0;
      B.p = 0;
      B.timestep = HUGE;
    }
    for (size_t i = 0; i < g_cells.size(); i++) {
      for (int term = 0; term < NTERM; term++) {
        g_cells[i].L[term] = 0;
        g_cells[i].M[term] = 0;
      }
      g_cells[i].min_acc = HUGE;
      g_cells[i].has_sink = false;
    }
    upwardPass(g_cells);
    for (size_t i = 0; i < g_cells.size(); i++)
      for (int nn = 0; nn <= P; nn++) {
        for (int mm = -nn; mm <= nn; mm++) {
          int index = nn * nn + nn + mm;
          g_cells[i].Pn[nn] += g_cells[i].M[index] * g_cells[i].M[index] * factorial_table[nn + mm] *
                               factorial_table[nn - mm];
        }
        g_cells[i].Pn[nn] = sqrt(g_cells[i].Pn[nn]);
      }
  } else
#endif
  {
    for (size_t c = 0; c < g_cells.size(); c++) g_cells[c].has_sink = false;
    upwardPass(g_cells);
  }
  double t2 = now_s();
  horizontalPass(g_cells, g_cells, high ? 1 : 0, get_steps);
  double t3 = now_s();
  downwardPass(g_cells);
  double t4 = now_s();
  if (times) {
    times[0] = t1 - t0; times[1] = t2 - t1; times[2] = t3 - t2; times[3] = t4 - t3;
  }
  for (int b = 0; b < n; b++) {
    const Body& B = bodies[b];
    int i = B.index;
    ax[i] = B.F[0]; ay[i] = B.F[1]; az[i] = B.F[2]; pot[i] = B.p;
    if (timestep) timestep[i] = B.timestep;
#ifdef TCR_JERKS
    if (jx) { jx[i] = B.J[0]; jy[i] = B.J[1]; jz[i] = B.J[2]; }
#else
    if (jx) { jx[i] = 0; jy[i] = 0; jz[i] = 0; }
#endif
  }
  for (int k = 0; k < 2; k++) { g_list_t[k].clear(); g_list_s[k].clear(); }
  return (int)g_cells.size();
}

extern "C" {

// Cells of the last evaluation in the reference's own order.
void tcr_cells(int* begin, int* nbody, int* nchild, int* child, double* X, double* R, int* index) {
  Body* b0 = &bodies[0];
  for (size_t c = 0; c < g_cells.size(); c++) {
    const Cell& C = g_cells[c];
    begin[c] = (int)(C.BODY - b0);
    nbody[c] = C.NBODY;
    nchild[c] = C.NCHILD;
    child[c] = C.NCHILD ? (int)(C.CHILD - &g_cells[0]) : -1;
    for (int d = 0; d < 3; d++) X[3 * c + d] = C.X[d];
    R[c] = C.R;
  }
  if (index)
    for (size_t i = 0; i < bodies.size(); i++) index[i] = bodies[i].index;
}

// per body acc_old of the last evaluation (caller order) and per cell min_acc, Pn[0..P]
void tcr_acc_old(double* out) {
  for (size_t b = 0; b < bodies.size(); b++) out[bodies[b].index] = bodies[b].acc_old;
}
void tcr_min_acc(double* out, double* pn) {
  for (size_t c = 0; c < g_cells.size(); c++) {
    out[c] = g_cells[c].min_acc;
    if (pn)
      for (int k = 0; k <= P; k++) pn[c * (P + 1) + k] = g_cells[c].Pn[k];
  }
}

void tcr_expansions(double* M, double* L) {
  for (size_t c = 0; c < g_cells.size(); c++) {
    memcpy(M + c * NTERM, g_cells[c].M, NTERM * sizeof(double));
    memcpy(L + c * NTERM, g_cells[c].L, NTERM * sizeof(double));
  }
}

// kind 0 = M2L, 1 = P2P.  First call with tgt == NULL walks the tree and returns the count.
long long tcr_list(int kind, int* tgt, int* src) {
  if (g_list_t[0].empty() && g_list_t[1].empty() && g_high) record_high(&g_cells[0], &g_cells[0]);
  if (g_list_t[0].empty() && g_list_t[1].empty()) record(&g_cells[0], &g_cells[0]);
  long long n = (long long)g_list_t[kind].size();
  if (tgt) memcpy(tgt, g_list_t[kind].data(), n * sizeof(int));
  if (src) memcpy(src, g_list_s[kind].data(), n * sizeof(int));
  return n;
}

}  // extern "C"
