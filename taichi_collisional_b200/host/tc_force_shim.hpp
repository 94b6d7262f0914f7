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
// get_steps == true (the pairwise time-step criterion of P2P, kernel_fast_lean.h:548-574) is
// not provided by the library; the shim stops the run with the reference's ENDRUN.
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
  if (get_steps) ENDRUN("get_force_and_potential(get_steps=true) is not provided by taichi_b200\n");
  const int n = (int)bodies.size();
  std::vector<double> x(n), y(n), z(n), vx(n), vy(n), vz(n), m(n), ax(n), ay(n), az(n), pot(n), jx(n), jy(n),
      jz(n);
  std::vector<unsigned char> flags(n);
  for (int i = 0; i < n; i++) {
    const Body& b = bodies[i];
    x[i] = b.X[0]; y[i] = b.X[1]; z[i] = b.X[2];
    vx[i] = b.V[0]; vy[i] = b.V[1]; vz[i] = b.V[2];
    m[i] = b.q;
    flags[i] = (unsigned char)((b.issink ? 1 : 0) | (b.issource ? 2 : 0));
  }
  tc_status s = tc_evaluate(tc_shim_context(), n, x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data(),
                            m.data(), flags.data(), ax.data(), ay.data(), az.data(), pot.data(), jx.data(),
                            jy.data(), jz.data(), TC_MEM_HOST);
  if (s != TC_OK) ENDRUN("tc_evaluate: %s\n", tc_status_string(s));
  for (int i = 0; i < n; i++) {
    Body& b = bodies[i];
    // the reference's FMM branch resets F, p (and J) before accumulating
    // (integrator.h:500-507, taichi_with_jerks/integrator.h:352-364)
    b.F[0] = ax[i]; b.F[1] = ay[i]; b.F[2] = az[i];
    b.p = pot[i];
#ifdef TC_SHIM_JERKS
    b.J[0] = jx[i]; b.J[1] = jy[i]; b.J[2] = jz[i];
#endif
  }
}

}  // namespace exafmm
