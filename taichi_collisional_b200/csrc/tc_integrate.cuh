// Block-time-step integrator of the reference, device-resident:
//   evolve_split_hold_dkd (integrator.h:834-871), called as do_evolve does (integrator.h:873-890),
// with its pieces
//   split by time step (integrator.h:591-640)                      -> k_split_* below,
//   kick_naive with update_timestep (integrator.h:182-311)        -> tc_evaluate_steps + k_ev_naive,
//   kick of sinks by sources (integrator.h:378-457)                -> tc_evaluate with flags + k_ev_kick,
//   kick_cpu, the direct kick of small systems (integrator.h:65-96) -> direct sums + k_ev_kick,
//   drift with COMPSUM (integrator.h:42, :642-656)                 -> k_drift_compsum.
// The particles stay in the caller's device arrays, which are permuted in place exactly as the
// reference's split swaps its particles, so after a step the arrays hold the reference's order
// (id[] tells which body is where).  The recursion itself runs on the host, one level per
// call, as in the reference; only the split's two counts are read back.
#pragma once

namespace tc {

// counts[k] = 1 if body k is fast (timestep < |dt|)
__global__ void k_split_mark(int ns, const double* __restrict__ ts, double adt, uint32_t* __restrict__ cnt) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < ns) cnt[k] = ts[k] < adt ? 1u : 0u;
}

// After the exclusive scan of the marks: nf = number of fast bodies, nswap = slow bodies in the
// fast prefix [0, nf) (= fast bodies in the slow suffix), out[0..1].
__global__ void k_split_count(int ns, const double* __restrict__ ts, double adt, const uint32_t* __restrict__ cnt,
                              int* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int nf = (int)cnt[ns - 1] + (ts[ns - 1] < adt ? 1 : 0);
  const int fast_in_prefix = nf < ns ? (int)cnt[nf] : nf;
  out[0] = nf;
  out[1] = nf - fast_in_prefix;
}

// The reference's two pointers swap the r-th slow body of the prefix (left to right) with the
// r-th fast body of the suffix (right to left): posL[r], posR[r].
__global__ void k_split_pairs(int ns, int nf, const double* __restrict__ ts, double adt,
                              const uint32_t* __restrict__ cnt, int* __restrict__ posL, int* __restrict__ posR) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  const bool fast = ts[k] < adt;
  const int c = (int)cnt[k];  // fast bodies in [0, k)
  if (k < nf && !fast) posL[k - c] = k;
  if (k >= nf && fast) posR[nf - c - 1] = k;
}

struct TcEvArrays {
  double* d[15];  // x y z ex ey ez vx vy vz m timestep pot (+ acc x y z for the gradient scheme)
  int nd;         // how many of d travel with the particles (12, or 15 with acc)
  int* id;
};

__global__ void k_split_swap(int nswap, TcEvArrays a, const int* __restrict__ posL, const int* __restrict__ posR) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nswap) return;
  const int L = posL[r], R = posR[r];
#pragma unroll
  for (int q = 0; q < 15; q++) {
    if (q >= a.nd) break;
    const double t = a.d[q][L];
    a.d[q][L] = a.d[q][R];
    a.d[q][R] = t;
  }
  const int t = a.id[L];
  a.id[L] = a.id[R];
  a.id[R] = t;
}

__global__ void k_split_perm(int ns, int* __restrict__ perm) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < ns) perm[k] = k;
}

__global__ void k_split_perm_swap(int nswap, const int* __restrict__ posL, const int* __restrict__ posR,
                                  int* __restrict__ perm) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nswap) return;
  perm[posL[r]] = posR[r];
  perm[posR[r]] = posL[r];
}

// flags of a kick on [0, ns): bodies [0, nf) get fa, [nf, ns) get fb (bit 0 sink, bit 1 source)
__global__ void k_ev_flags(int ns, int nf, uint8_t fa, uint8_t fb, uint8_t* __restrict__ fl) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < ns) fl[k] = k < nf ? fa : fb;
}

// kick_naive's update: timestep = 1 / sqrt(sqrt(sum 1/tau^4)), pot (its velocity kick has dt = 0)
__global__ void k_ev_naive(int ns, const double* __restrict__ tsum, const double* __restrict__ apot,
                           double* __restrict__ ts, double* __restrict__ pot) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  ts[k] = 1.0 / sqrt(sqrt(tsum[k]));
  pot[k] = apot[k];
}

// v += a dt for the sinks [k0, k1) of a kick; pot as well when set_pot (kick, not kick_cpu)
__global__ void k_ev_kick(int k0, int k1, const double* __restrict__ ax, const double* __restrict__ ay,
                          const double* __restrict__ az, const double* __restrict__ apot, double* __restrict__ vx,
                          double* __restrict__ vy, double* __restrict__ vz, double* __restrict__ pot, double dt,
                          int set_pot) {
  const int k = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k1) return;
  vx[k] = __fma_rn(ax[k], dt, vx[k]);
  vy[k] = __fma_rn(ay[k], dt, vy[k]);
  vz[k] = __fma_rn(az[k], dt, vz[k]);
  if (set_pot) pot[k] = apot[k];
}

__global__ void k_ev_zero_pot(int nk, double* __restrict__ pot) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nk) pot[k] = 0.0;
}

// The GRADIENT build of kick_naive (integrator.h:254-299): every sink's time step becomes the
// least over the system, 1 / sqrt(sqrt(sum 1/tau^4)) minimised (HUGE when every sum is 0), and
// (OUTPUTACC) its acc the pass's force.  Time steps are >= 0, so their bit patterns order as
// the values do and one atomicMin finds the least.
__global__ void k_ev_ts_min(int ns, const double* __restrict__ tsum, unsigned long long* __restrict__ mn) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < ns) atomicMin(mn, (unsigned long long)__double_as_longlong(1.0 / sqrt(sqrt(tsum[k]))));
}
__global__ void k_ev_naive_grad(int ns, const double* __restrict__ ax, const double* __restrict__ ay,
                                const double* __restrict__ az, const double* __restrict__ apot,
                                const unsigned long long* __restrict__ mn, double* __restrict__ ts,
                                double* __restrict__ pot, double* __restrict__ accx, double* __restrict__ accy,
                                double* __restrict__ accz) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  ts[k] = __longlong_as_double((long long)*mn);
  pot[k] = apot[k];
  accx[k] = ax[k];
  accy[k] = ay[k];
  accz[k] = az[k];
}

// kick_gradient's positions (integrator.h:313-351): X = pos + acc dt^2 / 24
__global__ void k_ev_shift(int ns, const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, const double* __restrict__ accx,
                           const double* __restrict__ accy, const double* __restrict__ accz, double fac,
                           double* __restrict__ xs, double* __restrict__ ys, double* __restrict__ zs) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  xs[k] = x[k] + accx[k] * fac;
  ys[k] = y[k] + accy[k] * fac;
  zs[k] = z[k] + accz[k] * fac;
}

__global__ void k_ev_set_u64(unsigned long long* p, unsigned long long v) { *p = v; }

struct TcEvolve {
  tc_ctx* ctx;
  TcEvArrays a;
  double dt_param;
  double *ax, *ay, *az, *apot, *tsum;
  double *xs, *ys, *zs;    // kick_gradient's shifted positions (gradient scheme only)
  unsigned long long* mn;  // the least time step of a GRADIENT kick_naive (bit pattern)
  uint32_t* cnt;
  uint32_t* sums;
  int *posL, *posR, *small;
  uint8_t* fl;
  tc_evolve_stats st;

  double* X(int q, int off) const { return a.d[q] + off; }

  tc_status naive(int off, int ns) {
    const cudaStream_t s = ctx->stream;
    tc_status r = tc_evaluate_steps(ctx, ns, X(0, off), X(1, off), X(2, off), X(6, off), X(7, off), X(8, off),
                                    X(9, off), nullptr, dt_param, ax, ay, az, apot, tsum, TC_MEM_DEVICE);
    if (r != TC_OK) return r;
    k_ev_naive<<<nblocks(ns, 256), 256, 0, s>>>(ns, tsum, apot, X(10, off), X(11, off));
    st.n_evaluations++;
    return cudaGetLastError() == cudaSuccess ? TC_OK : TC_ERR_CUDA;
  }

  // kick of [k0, k1) (sinks) with the flags already in fl over the system [off, off + ns)
  tc_status kick(int off, int ns, int k0, int k1, double dt, bool direct) {
    const cudaStream_t s = ctx->stream;
    tc_status r;
    if (direct) {
      // the context's own storage (never the library-wide static array of
      // tc_evaluate_direct_noalloc, which contexts stepping at once would share)
      const size_t S = ctx->kd_cap;
      r = (size_t)ns <= S && direct_with_scratch(ns, X(0, off), X(1, off), X(2, off), nullptr, nullptr, nullptr,
                                                 X(9, off), fl, ax, ay, az, apot, nullptr, nullptr, nullptr, 0, s,
                                                 ctx->kd_scratch.p, ctx->kd_index.p, ctx->kd_flags.p, S,
                                                 ctx->prm.softening * ctx->prm.softening) == cudaSuccess
              ? TC_OK
              : TC_ERR_CUDA;
      st.n_direct++;
    } else {
      r = tc_evaluate(ctx, ns, X(0, off), X(1, off), X(2, off), nullptr, nullptr, nullptr, X(9, off), fl, ax, ay, az,
                      apot, nullptr, nullptr, nullptr, TC_MEM_DEVICE);
      st.n_evaluations++;
    }
    if (r != TC_OK) return r;
    if (k1 > k0)
      k_ev_kick<<<nblocks(k1 - k0, 256), 256, 0, s>>>(k0, k1, ax, ay, az, apot, X(6, off), X(7, off), X(8, off),
                                                      X(11, off), dt, direct ? 0 : 1);
    return cudaGetLastError() == cudaSuccess ? TC_OK : TC_ERR_CUDA;
  }

  void flags(int ns, int nf, uint8_t fa, uint8_t fb) {
    k_ev_flags<<<nblocks(ns, 256), 256, 0, ctx->stream>>>(ns, nf, fa, fb, fl);
  }

  tc_status drift(int off, int ns, double dt) {
    if (ns <= 0) return TC_OK;
    k_drift_compsum<<<nblocks(ns, 256), 256, 0, ctx->stream>>>(ns, X(0, off), X(1, off), X(2, off), X(3, off),
                                                              X(4, off), X(5, off), X(6, off), X(7, off), X(8, off),
                                                              dt);
    return cudaGetLastError() == cudaSuccess ? TC_OK : TC_ERR_CUDA;
  }

  // split(dt, s, &slow, &fast): permutes [off, off + ns) in place; returns fast.n (0 for one)
  tc_status split(int off, int ns, double dt, int* nfast) {
    const cudaStream_t s = ctx->stream;
    const double adt = fabs(dt);
    const double* ts = a.d[10] + off;
    k_split_mark<<<nblocks(ns, 256), 256, 0, s>>>(ns, ts, adt, cnt);
    excl_scan(cnt, ns, sums, s);
    k_split_count<<<1, 32, 0, s>>>(ns, ts, adt, cnt, small);
    int h[2];
    if (cudaMemcpyAsync(h, small, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return TC_ERR_CUDA;
    const int nf = h[0], nswap = h[1];
    if (nswap > 0) {
      k_split_pairs<<<nblocks(ns, 256), 256, 0, s>>>(ns, nf, ts, adt, cnt, posL, posR);
      TcEvArrays sub = a;
      for (int q = 0; q < a.nd; q++) sub.d[q] += off;
      sub.id += off;
      k_split_swap<<<nblocks(nswap, 256), 256, 0, s>>>(nswap, sub, posL, posR);
    }
    st.n_splits++;
    *nfast = nf == 1 ? 0 : nf;
    return cudaGetLastError() == cudaSuccess ? TC_OK : TC_ERR_CUDA;
  }

  // evolve_split_hold_dkd(clevel, s, stime, etime, dt, calc_timestep) on s = [off, off + ns)
  tc_status hold_dkd(int clevel, int off, int ns, double dt, bool calc_timestep) {
    if (clevel > kMaxLevelEvolve) {
      ctx->err = "time-step hierarchy deeper than 64 levels (a time step is zero or not finite)";
      return TC_ERR_ARG;
    }
    st.max_level = std::max(st.max_level, clevel);
    tc_status r;
    if (calc_timestep && (r = naive(off, ns)) != TC_OK) return r;
    int nf = 0;
    if ((r = split(off, ns, dt, &nf)) != TC_OK) return r;
    const int nslow = ns - nf;
    if (nf == 0) st.simtime += dt;
    if (nf > 0 && (r = hold_dkd(clevel + 1, off, nf, dt / 2, false)) != TC_OK) return r;
    if ((r = drift(off + nf, nslow, dt / 2)) != TC_OK) return r;
    if (ns > 128) {
      if (nslow > 0) {
        flags(ns, nf, 2, 3);  // kick(slow, fast, dt, sinks_are_fast = false)
        if ((r = kick(off, ns, nf, ns, dt, false)) != TC_OK) return r;
      }
      if (nf > 0 && nslow > 0) {
        flags(ns, nf, 1, 2);  // kick(fast, slow, dt, sinks_are_fast = true)
        if ((r = kick(off, ns, 0, nf, dt, false)) != TC_OK) return r;
      } else if (nf > 0) {
        // kick(fast, slow) with no slow body: no source, so F = 0 and p = 0 for the fast sinks
        k_ev_zero_pot<<<nblocks(nf, 256), 256, 0, ctx->stream>>>(nf, X(11, off));
      }
    } else if (nslow > 0) {
      flags(ns, nf, 2, 3);  // kick_cpu(slow, join(slow, fast), dt)
      if ((r = kick(off, ns, nf, ns, dt, true)) != TC_OK) return r;
      if (nf > 0) {
        flags(ns, nf, 1, 2);  // kick_cpu(fast, slow, dt)
        if ((r = kick(off, ns, 0, nf, dt, true)) != TC_OK) return r;
      }
    }
    if ((r = drift(off + nf, nslow, dt / 2)) != TC_OK) return r;
    if (nf > 0 && (r = hold_dkd(clevel + 1, off, nf, dt / 2, true)) != TC_OK) return r;
    return TC_OK;
  }
  // kick_naive(clevel, s, 0, 0, 0, true) as the GRADIENT build runs it (integrator.h:254-299)
  tc_status naive_grad(int off, int ns) {
    const cudaStream_t s = ctx->stream;
    tc_status r = tc_evaluate_steps(ctx, ns, X(0, off), X(1, off), X(2, off), X(6, off), X(7, off), X(8, off),
                                    X(9, off), nullptr, dt_param, ax, ay, az, apot, tsum, TC_MEM_DEVICE);
    if (r != TC_OK) return r;
    k_ev_set_u64<<<1, 1, 0, s>>>(mn, 0x7FF0000000000000ull);  // +inf (HUGE_VAL)
    k_ev_ts_min<<<nblocks(ns, 256), 256, 0, s>>>(ns, tsum, mn);
    k_ev_naive_grad<<<nblocks(ns, 256), 256, 0, s>>>(ns, ax, ay, az, apot, mn, X(10, off), X(11, off), X(12, off),
                                                     X(13, off), X(14, off));
    st.n_evaluations++;
    return cudaGetLastError() == cudaSuccess ? TC_OK : TC_ERR_CUDA;
  }

  // kick_gradient (integrator.h:313-376) of [k0, k1) with the flags in fl over [off, off + ns):
  // the forces at X = pos + acc dt^2 / 24, then v += F 2 dt / 3.  The reference then stores an
  // uninitialised array as the potential; the potential is left as the last kick set it.
  tc_status gkick(int off, int ns, int k0, int k1, double dt) {
    const cudaStream_t s = ctx->stream;
    k_ev_shift<<<nblocks(ns, 256), 256, 0, s>>>(ns, X(0, off), X(1, off), X(2, off), X(12, off), X(13, off),
                                                X(14, off), dt * dt / 24.0, xs, ys, zs);
    tc_status r = tc_evaluate(ctx, ns, xs, ys, zs, nullptr, nullptr, nullptr, X(9, off), fl, ax, ay, az, apot, nullptr,
                              nullptr, nullptr, TC_MEM_DEVICE);
    st.n_evaluations++;
    if (r != TC_OK) return r;
    if (k1 > k0)
      k_ev_kick<<<nblocks(k1 - k0, 256), 256, 0, s>>>(k0, k1, ax, ay, az, apot, X(6, off), X(7, off), X(8, off),
                                                      X(11, off), dt * 2.0 / 3.0, 0);
    return cudaGetLastError() == cudaSuccess ? TC_OK : TC_ERR_CUDA;
  }

  // the dt / 6 kicks that open and close evolve_split_omelyan (integrator.h:741-754, :797-811)
  tc_status omelyan_outer(int off, int ns, int nf, double dtk) {
    const int nslow = ns - nf;
    tc_status r;
    if (ns > 128) {
      if (nslow > 0) {
        flags(ns, nf, 2, 3);  // kick(slow, fast, dt / 6, sinks_are_fast = false)
        if ((r = kick(off, ns, nf, ns, dtk, false)) != TC_OK) return r;
      }
      if (nf > 0 && nslow > 0) {
        flags(ns, nf, 1, 2);  // kick(fast, slow, dt / 6, sinks_are_fast = true)
        if ((r = kick(off, ns, 0, nf, dtk, false)) != TC_OK) return r;
      } else if (nf > 0) {
        k_ev_zero_pot<<<nblocks(nf, 256), 256, 0, ctx->stream>>>(nf, X(11, off));  // no source: F = 0, p = 0
      }
    } else if (nslow > 0) {
      flags(ns, nf, 2, 3);  // kick_cpu(slow, join(slow, fast), dt / 6)
      if ((r = kick(off, ns, nf, ns, dtk, true)) != TC_OK) return r;
      if (nf > 0) {
        flags(ns, nf, 1, 2);  // kick_cpu(fast, slow, dt / 6)
        if ((r = kick(off, ns, 0, nf, dtk, true)) != TC_OK) return r;
      }
    }
    return TC_OK;
  }

  // evolve_split_omelyan(clevel, s, stime, etime, dt, calc_timestep) (integrator.h:720-812), the
  // force-gradient scheme of the reference's default build (GRADIENT, OUTPUTACC), on
  // s = [off, off + ns)
  tc_status omelyan(int clevel, int off, int ns, double dt, bool calc_timestep) {
    if (clevel > kMaxLevelEvolve) {
      ctx->err = "time-step hierarchy deeper than 64 levels (a time step is zero or not finite)";
      return TC_ERR_ARG;
    }
    st.max_level = std::max(st.max_level, clevel);
    tc_status r;
    if (calc_timestep && (r = naive_grad(off, ns)) != TC_OK) return r;
    int nf = 0;
    if ((r = split(off, ns, dt, &nf)) != TC_OK) return r;
    const int nslow = ns - nf;
    if (nf == 0) st.simtime += dt;
    if ((r = omelyan_outer(off, ns, nf, dt / 6)) != TC_OK) return r;
    if (nf > 0 && (r = omelyan(clevel + 1, off, nf, dt / 2, false)) != TC_OK) return r;
    if ((r = drift(off + nf, nslow, dt / 2)) != TC_OK) return r;
    // the middle: zero-length kicks that set the potential, then the gradient kicks (2 dt / 3)
    // with the positions shifted by the acc of the last kick_naive
    if (nslow > 0) {
      flags(nslow, 0, 3, 3);  // kick(slow, zerosys, 0): the slow bodies alone
      if ((r = kick(off + nf, nslow, 0, nslow, 0.0, false)) != TC_OK) return r;
      flags(nslow, 0, 3, 3);  // kick_gradient(slow, zerosys, dt)
      if ((r = gkick(off + nf, nslow, 0, nslow, dt)) != TC_OK) return r;
      if (nf > 0) {
        flags(ns, nf, 2, 1);  // kick(slow, fast, 0, sinks_are_fast = true)
        if ((r = kick(off, ns, nf, ns, 0.0, false)) != TC_OK) return r;
      } else {
        k_ev_zero_pot<<<nblocks(nslow, 256), 256, 0, ctx->stream>>>(nslow, X(11, off + nf));
      }
    }
    if (nf > 0) {
      if (nslow > 0) {
        flags(ns, nf, 1, 2);  // kick(fast, slow, 0, sinks_are_fast = true)
        if ((r = kick(off, ns, 0, nf, 0.0, false)) != TC_OK) return r;
      } else {
        k_ev_zero_pot<<<nblocks(nf, 256), 256, 0, ctx->stream>>>(nf, X(11, off));
      }
    }
    if (nslow > 0 && nf > 0) {
      flags(ns, nf, 2, 1);  // kick_gradient(slow, fast, dt, true)
      if ((r = gkick(off, ns, nf, ns, dt)) != TC_OK) return r;
      flags(ns, nf, 1, 2);  // kick_gradient(fast, slow, dt, true)
      if ((r = gkick(off, ns, 0, nf, dt)) != TC_OK) return r;
    }
    if ((r = drift(off + nf, nslow, dt / 2)) != TC_OK) return r;
    if (nf > 0 && (r = omelyan(clevel + 1, off, nf, dt / 2, true)) != TC_OK) return r;
    return omelyan_outer(off, ns, nf, dt / 6);
  }
  static constexpr int kMaxLevelEvolve = 64;  // MAXLEVEL, integrator.h:8
};

}  // namespace tc

extern "C" tc_status tc_split_order(tc_ctx* ctx, int n, const double* timestep, double dt, int* perm, int* nfast) {
  using namespace tc;
  if (!ctx || n <= 0 || !timestep || !perm || !nfast) return TC_ERR_ARG;
  TC_CK(cudaSetDevice(ctx->prm.device));
  TC_CK(ctx->ev_u.ensure((size_t)n + (size_t)n / 4096 + 2));
  TC_CK(ctx->ev_i.ensure(2 * (size_t)n + 2));
  const cudaStream_t s = ctx->stream;
  const double adt = fabs(dt);
  uint32_t* cnt = ctx->ev_u.p;
  int *posL = ctx->ev_i.p, *posR = posL + n, *small = posR + n;
  k_split_mark<<<nblocks(n, 256), 256, 0, s>>>(n, timestep, adt, cnt);
  excl_scan(cnt, n, cnt + n, s);
  k_split_count<<<1, 32, 0, s>>>(n, timestep, adt, cnt, small);
  int h[2];
  TC_CK(cudaMemcpyAsync(h, small, sizeof(h), cudaMemcpyDeviceToHost, s));
  TC_CK(cudaStreamSynchronize(s));
  k_split_perm<<<nblocks(n, 256), 256, 0, s>>>(n, perm);
  if (h[1] > 0) {
    k_split_pairs<<<nblocks(n, 256), 256, 0, s>>>(n, h[0], timestep, adt, cnt, posL, posR);
    k_split_perm_swap<<<nblocks(h[1], 256), 256, 0, s>>>(h[1], posL, posR, perm);
  }
  TC_CK(cudaGetLastError());
  TC_CK(cudaStreamSynchronize(s));
  *nfast = h[0] == 1 ? 0 : h[0];
  return TC_OK;
}

namespace tc {
// one do_evolve(s, dt) (integrator.h:873-890) of the HOLD (gradient = false) or the GRADIENT scheme
static tc_status tc_evolve_run(tc_ctx* ctx, int n, double* x, double* y, double* z, double* ex, double* ey,
                               double* ez, double* vx, double* vy, double* vz, double* m, double* timestep,
                               double* pot, int* id, double dt_param, double dt, tc_evolve_stats* st, bool gradient) {
  if (!ctx || n <= 0 || !x || !y || !z || !ex || !ey || !ez || !vx || !vy || !vz || !m || !timestep || !pot || !id ||
      !(dt != 0.0) || !std::isfinite(dt))
    return TC_ERR_ARG;
  if (ctx->prm.variant != TC_VARIANT_TOP) {
    ctx->err = "the block-time-step integrator drives the top-level tree (the jerks tree has no time-step pass)";
    return TC_ERR_UNSUPPORTED;
  }
  TC_CK(cudaSetDevice(ctx->prm.device));
  TC_CK(ctx->ev_d.ensure((gradient ? 11 : 5) * (size_t)n));
  // marks and scan sums (n + n / 4096 + 2), then the 8-byte least time step on an even index
  const size_t mn_at = ((size_t)n + (size_t)n / 4096 + 3) & ~(size_t)1;
  TC_CK(ctx->ev_u.ensure(mn_at + 2));
  TC_CK(ctx->ev_i.ensure(2 * (size_t)n + 2));
  TC_CK(ctx->ev_f.ensure((size_t)n));
  // systems of at most kDirectMax bodies are kicked by direct sums (kick_cpu)
  constexpr size_t kDirectMax = 128;
  TC_CK(ctx->kd_scratch.ensure(14 * kDirectMax));
  TC_CK(ctx->kd_index.ensure(kDirectMax));
  TC_CK(ctx->kd_flags.ensure(kDirectMax));
  ctx->kd_cap = kDirectMax;
  TcEvolve E;
  E.ctx = ctx;
  double* arr[12] = {x, y, z, ex, ey, ez, vx, vy, vz, m, timestep, pot};
  for (int q = 0; q < 12; q++) E.a.d[q] = arr[q];
  E.a.nd = 12;
  E.a.id = id;
  E.dt_param = dt_param;
  E.ax = ctx->ev_d.p; E.ay = E.ax + n; E.az = E.ay + n; E.apot = E.az + n; E.tsum = E.apot + n;
  E.xs = E.ys = E.zs = nullptr;
  if (gradient) {
    // the particles' acc (OUTPUTACC) travels with them through the splits
    E.a.d[12] = E.tsum + n; E.a.d[13] = E.a.d[12] + n; E.a.d[14] = E.a.d[13] + n;
    E.a.nd = 15;
    E.xs = E.a.d[14] + n; E.ys = E.xs + n; E.zs = E.ys + n;
  }
  E.cnt = ctx->ev_u.p; E.sums = E.cnt + n;
  E.mn = (unsigned long long*)(ctx->ev_u.p + mn_at);
  E.posL = ctx->ev_i.p; E.posR = E.posL + n; E.small = E.posR + n;
  E.fl = ctx->ev_f.p;
  E.st = tc_evolve_stats{};
  // do_evolve (integrator.h:873-890): kick_naive(0, s, 0, 0, 0, true), then the scheme with
  // calc_timestep = true, whose first act is the same kick_naive on the same state; the
  // result of the first is overwritten unchanged by the second, so it is done once.
  tc_status r = gradient ? E.omelyan(0, 0, n, dt, true) : E.hold_dkd(0, 0, n, dt, true);
  if (r == TC_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) r = TC_ERR_CUDA;
  if (st) *st = E.st;
  return r;
}
}  // namespace tc

extern "C" tc_status tc_evolve_hold_dkd(tc_ctx* ctx, int n, double* x, double* y, double* z, double* ex, double* ey,
                                        double* ez, double* vx, double* vy, double* vz, double* m, double* timestep,
                                        double* pot, int* id, double dt_param, double dt, tc_evolve_stats* st) {
  return tc::tc_evolve_run(ctx, n, x, y, z, ex, ey, ez, vx, vy, vz, m, timestep, pot, id, dt_param, dt, st, false);
}

extern "C" tc_status tc_evolve_omelyan(tc_ctx* ctx, int n, double* x, double* y, double* z, double* ex, double* ey,
                                       double* ez, double* vx, double* vy, double* vz, double* m, double* timestep,
                                       double* pot, int* id, double dt_param, double dt, tc_evolve_stats* st) {
  return tc::tc_evolve_run(ctx, n, x, y, z, ex, ey, ez, vx, vy, vz, m, timestep, pot, id, dt_param, dt, st, true);
}
