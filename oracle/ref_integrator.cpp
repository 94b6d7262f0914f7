// Harness around the reference's integrator (integrator.h) -- TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/Makefile against the reference sources where they lie (nothing is copied
// into this repository) into oracle/_ref/libtcref_integ_<isa>.so.  It exposes, on plain
// arrays, the reference's own
//   system_kinetic_energy / system_potential_energy / system_center_of_mass (integrator.h:887-925),
//   drift with COMPSUM (integrator.h:42, :642-656),
//   split by time step (integrator.h:591-640),
//   one do_evolve step (integrator.h:873-890) of the HOLD scheme evolve_split_hold_dkd
//   (integrator.h:834-871) with the reference's own force evaluation (error-controlled MAC) --
//   or, in a build with GRADIENT and OUTPUTACC, of the force-gradient scheme
//   evolve_split_omelyan (integrator.h:720-812),
// so the oracle's restatements and the CUDA kernels can be pinned against them.  The same
// source, compiled with TCR_SHIM, drives the reference's integrator over this repository's
// force evaluation instead (taichi_collisional_b200/host/tc_force_shim.hpp): the Makefile then
// feeds it a copy of integrator.h, generated into oracle/_ref/, without the reference's own
// get_force_and_potential (the step the shim's integration recipe asks for).
#include <cmath>
#include <cstring>
#include <list>
#include <vector>

#include "exafmm.h"
#ifdef TCR_SHIM
#define TC_SHIM_ERROR_MAC
#include "taichi_collisional_b200/host/tc_force_shim.hpp"
#include "integrator_noforce.h"
#else
#include "integrator.h"
#endif

struct sys zerosys = {0, NULL, NULL};
struct diagnostics global_diag;
struct diagnostics* diag = &global_diag;

static std::vector<particle> make_parts(int n, const double* m, const double* x, const double* y, const double* z,
                                        const double* vx, const double* vy, const double* vz) {
  std::vector<particle> p(n);
  for (int i = 0; i < n; i++) {
    memset(&p[i], 0, sizeof(particle));
    p[i].mass = m ? m[i] : 0;
    p[i].pos[0] = x ? x[i] : 0; p[i].pos[1] = y ? y[i] : 0; p[i].pos[2] = z ? z[i] : 0;
    p[i].vel[0] = vx ? vx[i] : 0; p[i].vel[1] = vy ? vy[i] : 0; p[i].vel[2] = vz ? vz[i] : 0;
    p[i].id = i;
  }
  return p;
}

extern "C" {

void tcr_system_diagnostics(int n, const double* m, const double* x, const double* y, const double* z,
                            const double* vx, const double* vy, const double* vz, const double* pot, double* out) {
  std::vector<particle> p = make_parts(n, m, x, y, z, vx, vy, vz);
  for (int i = 0; i < n; i++) p[i].pot = pot[i];
  struct sys s = {(size_t)n, p.data(), p.data() + n - 1};
  out[0] = system_kinetic_energy(s);
  out[1] = system_potential_energy(s);
  long double cp[3], cv[3];
  system_center_of_mass(s, cp, cv);
  long double mass = 0;
  for (int i = 0; i < n; i++) mass += (long double)p[i].mass;
  out[2] = (double)mass;
  for (int d = 0; d < 3; d++) {
    out[3 + d] = (double)cp[d];
    out[6 + d] = (double)cv[d];
  }
}

// drift(clevel, s, etime, dt) on (x, y, z) with running errors (ex, ey, ez), in place
void tcr_drift(int n, double* x, double* y, double* z, double* ex, double* ey, double* ez, const double* vx,
               const double* vy, const double* vz, double dt) {
  std::vector<particle> p = make_parts(n, nullptr, x, y, z, vx, vy, vz);
  for (int i = 0; i < n; i++) {
    p[i].pos_e[0] = ex[i]; p[i].pos_e[1] = ey[i]; p[i].pos_e[2] = ez[i];
  }
  struct sys s = {(size_t)n, p.data(), p.data() + n - 1};
  drift(0, s, 0.0, dt);
  for (int i = 0; i < n; i++) {
    x[i] = p[i].pos[0]; y[i] = p[i].pos[1]; z[i] = p[i].pos[2];
    ex[i] = p[i].pos_e[0]; ey[i] = p[i].pos_e[1]; ez[i] = p[i].pos_e[2];
  }
}

// split(dt, s, &slow, &fast) on particles carrying timestep ts[i] and id i: writes the order
// the particles end in (perm[k] = id at position k) and returns fast.n (slow.n = n - fast.n)
int tcr_split(int n, const double* ts, double dt, int* perm) {
  std::vector<particle> p = make_parts(n, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  for (int i = 0; i < n; i++) p[i].timestep = ts[i];
  struct sys s = {(size_t)n, p.data(), p.data() + n - 1}, slow = zerosys, fast = zerosys;
  split(dt, s, &slow, &fast);
  for (int i = 0; i < n; i++) perm[i] = (int)p[i].id;
  return (int)fast.n;
}

// one do_evolve(mainsys, dt) of the build's scheme (HOLD, or GRADIENT) on n particles (arrays in
// and out, in the order the particles end in; id[] follows them); returns diag->simtime advanced
double tcr_evolve_hold(int n, double* x, double* y, double* z, double* ex, double* ey, double* ez, double* vx,
                       double* vy, double* vz, double* m, double* ts, double* pot, int* id, int nc, double th,
                       double fa, double dtp, double dt) {
  static bool init = false;
  if (!init) {
    P = EXPANSION;
#ifndef TCR_SHIM
    initKernel();
#endif
    init = true;
  }
  ncrit = nc;
  theta = th;
  force_accuracy = fa;
  dt_param = dtp;
  std::vector<particle> p = make_parts(n, m, x, y, z, vx, vy, vz);
  for (int i = 0; i < n; i++) {
    p[i].pos_e[0] = ex[i]; p[i].pos_e[1] = ey[i]; p[i].pos_e[2] = ez[i];
    p[i].timestep = ts[i];
    p[i].pot = pot[i];
    p[i].id = (unsigned)id[i];
  }
  mainsys.n = n;
  mainsys.part = p.data();
  mainsys.last = p.data() + n - 1;
  global_diag.simtime = 0;
  diag = &global_diag;
  do_evolve(mainsys, dt);
  for (int i = 0; i < n; i++) {
    x[i] = p[i].pos[0]; y[i] = p[i].pos[1]; z[i] = p[i].pos[2];
    ex[i] = p[i].pos_e[0]; ey[i] = p[i].pos_e[1]; ez[i] = p[i].pos_e[2];
    vx[i] = p[i].vel[0]; vy[i] = p[i].vel[1]; vz[i] = p[i].vel[2];
    m[i] = p[i].mass;
    ts[i] = p[i].timestep;
    pot[i] = p[i].pot;
    id[i] = (int)p[i].id;
  }
  return global_diag.simtime;
}

}  // extern "C"
