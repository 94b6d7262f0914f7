// Drop-in replacement of the reference's force evaluation on top of the C ABI.
//
// Include this header in the reference program instead of its FMM call path and link
// libtaichi_b200.so.  It defines
//
//   void exafmm::get_force_and_potential(Bodies& bodies, bool get_steps);
//
// with the contract of integrator.h:459-562 (top-level tree) or
// taichi_with_jerks/integrator.h:308-432 (jerks tree, when TC_SHIM_JERKS is defined):
//   reads  Body::X, q, V (jerks), issink, issource and the globals P, ncrit, theta;
//   writes Body::F (acceleration, G = 1), p (positive potential) and J (jerks),
// so kick_naive (integrator.h:182), kick_gradient (:313) and kick (:378) stay unchanged.
// Unlike the reference, `bodies` keeps its order (results are written in place, so the
// Body::index round trip still works but is no longer needed).
//
// Traversal: the jerks tree's get_force_and_potential always runs its low-order pre-pass and
// its one-sided error-controlled MAC (taichi_with_jerks/integrator.h:326-403,
// horizontalPass(cells, cells, 1, get_steps)), and so does the jerks shim, with the global
// force_accuracy (define TC_SHIM_THETA to use the theta MAC instead).  For the top-level tree
// the shim uses the theta MAC unless TC_SHIM_ERROR_MAC is defined, which selects the top
// tree's own pre-pass and error-controlled MAC (integrator.h:476-539).  With the error MAC,
// Body::acc_old receives the pre-pass's estimate as in the reference; otherwise (and on the
// direct-sum branch of small N) it is left unchanged.
//
// get_steps == true: for the top-level tree, the time-step pass of the reference
// (tc_evaluate_steps: no M2L, near-field F and p, Body::timestep = sum of 1/tau^4 from the
// pairwise criterion of kernel_fast_lean.h:462-548, with the global dt_param); the jerks
// tree's traversal ignores get_steps (taichi_with_jerks/traverse_eager.h:59-155), and so does
// the shim.  Body::timestep is otherwise reset as the reference does (0 for the top-level
// tree, integrator.h:500-507; HUGE for the jerks tree, taichi_with_jerks/integrator.h:352-364).
#pragma once
#include <vector>

#include "../../include/taichi_b200.h"

namespace exafmm {

inline tc_ctx* tc_shim_context() {
  static tc_ctx* ctx = nullptr;
  if (!ctx) {
    tc_params prm;
    tc_default_params(&prm);
    prm.p = P;
    prm.ncrit = ncrit;
    prm.theta = theta;
#ifdef TC_SHIM_JERKS
    prm.variant = TC_VARIANT_JERKS;
#else
    prm.variant = TC_VARIANT_TOP;
#endif
    prm.direct_below = -1;  // the reference's own small-N rule
    tc_status s = tc_create(&prm, &ctx);
    if (s != TC_OK) ENDRUN("tc_create: %s\n", tc_status_string(s));
  }
  return ctx;
}

inline void get_force_and_potential(Bodies& bodies, bool get_steps) {
#ifdef TC_SHIM_JERKS
  get_steps = false;
#endif
  const int n = (int)bodies.size();
  // an empty body list is a call the reference makes (the force-gradient scheme kicks an empty
  // slow system when every body is fast): nothing to evaluate
  if (n == 0) return;
  std::vector<double> x(n), y(n), z(n), vx(n), vy(n), vz(n), m(n), ax(n), ay(n), az(n), pot(n), jx(n), jy(n),
      jz(n), ts(n);
  std::vector<unsigned char> flags(n);
  for (int i = 0; i < n; i++) {
    const Body& b = bodies[i];
    x[i] = b.X[0]; y[i] = b.X[1]; z[i] = b.X[2];
    vx[i] = b.V[0]; vy[i] = b.V[1]; vz[i] = b.V[2];
    m[i] = b.q;
    flags[i] = (unsigned char)((b.issink ? 1 : 0) | (b.issource ? 2 : 0));
  }
  tc_status s;
#if (defined(TC_SHIM_ERROR_MAC) && !defined(TC_SHIM_JERKS)) || (defined(TC_SHIM_JERKS) && !defined(TC_SHIM_THETA))
#define TC_SHIM_USES_ERROR_MAC 1
  // the tree's own traversal: low-order pre-pass + error-controlled MAC with the current
  // global force_accuracy (integrator.h:459-562, taichi_with_jerks/integrator.h:308-432;
  // main.cxx changes force_accuracy for a while)
  s = tc_set_error_mac(tc_shim_context(), 1, force_accuracy);
  if (s != TC_OK) ENDRUN("tc_set_error_mac: %s\n", tc_status_string(s));
#endif
#ifndef TC_SHIM_JERKS
  if (get_steps)
    s = tc_evaluate_steps(tc_shim_context(), n, x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data(),
                          m.data(), flags.data(), dt_param, ax.data(), ay.data(), az.data(), pot.data(), ts.data(),
                          TC_MEM_HOST);
  else
#endif
    s = tc_evaluate(tc_shim_context(), n, x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data(), m.data(),
                    flags.data(), ax.data(), ay.data(), az.data(), pot.data(), jx.data(), jy.data(), jz.data(),
                    TC_MEM_HOST);
  if (s != TC_OK) ENDRUN("taichi_b200 force evaluation: %s\n", tc_status_string(s));
#ifdef TC_SHIM_USES_ERROR_MAC
  std::vector<double> acc_old(n);
  // TC_ERR_UNSUPPORTED on the direct-sum branch, which has no pre-pass: acc_old stays
  const bool have_acc_old = tc_get_acc_old(tc_shim_context(), acc_old.data()) == TC_OK;
#endif
  for (int i = 0; i < n; i++) {
    Body& b = bodies[i];
    // the reference's FMM branch resets F, p (and J) before accumulating
    // (integrator.h:500-507, taichi_with_jerks/integrator.h:352-364)
    b.F[0] = ax[i]; b.F[1] = ay[i]; b.F[2] = az[i];
    b.p = pot[i];
#ifdef TC_SHIM_USES_ERROR_MAC
    if (have_acc_old) b.acc_old = acc_old[i];
#endif
#ifdef TC_SHIM_JERKS
    b.J[0] = jx[i]; b.J[1] = jy[i]; b.J[2] = jz[i];
    b.timestep = HUGE;
#else
    b.timestep = get_steps ? ts[i] : 0;
#endif
  }
}

}  // namespace exafmm
