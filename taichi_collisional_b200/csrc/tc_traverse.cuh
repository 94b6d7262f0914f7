// Dual-tree traversal on the device: breadth-first expansion of (target, source) cell pairs.
// Each pair takes exactly the decision of the reference recursion (traverse_eager.h:151-203;
// taichi_with_jerks/traverse_eager.h:125-155):
//   |Xi - Xj|^2 theta^2 > (Ri + Rj)^2  -> M2L (top tree: P2P when one cell holds <= 2 and
//                                          the other <= 8 bodies, :160)
//   both leaves                        -> P2P
//   Cj leaf, or Ri >= Rj and Ci inner  -> (child of Ci, Cj) for every child
//   otherwise                          -> (Ci, child of Cj) for every child
// so the set of emitted pairs equals the set the recursion visits.  The emission order is
// not deterministic; the lists are radix-sorted by (target, source) afterwards.
#pragma once
#include "tc_common.cuh"

namespace tc {

// acceptance test of a traversal (mode 0: theta, traverse_eager.h:151-203; 1: the low-order
// pre-pass, |d|^2 > 3 (Ri + Rj)^2 on geometric cells, :220-245; 2: the top tree's error-
// controlled MAC of horizontalPassHigh, :61-148, with the reference's binomials comb[k] =
// combinator_coef[P][k]; 3: the jerks tree's one-sided horizontalPassHigh,
// taichi_with_jerks/traverse_eager.h:59-122)
struct TcMac {
  int mode = 0;
  int p = 0;
  double fa = 0.0;
  const double* pn = nullptr;       // (p + 1) per cell
  const double* min_acc = nullptr;  // per cell
  double comb[TC_PMAX_DEV + 1];
  // > 0: an accepted pair whose target is a leaf and whose body counts multiply to at most this
  // becomes a P2P pair (exact, and cheaper than its M2L); the order selectors' form only
  long long p2p_max = 0;
};

// x^-k correctly rounded (k >= 1): x^k in double-double by repeated products, then the
// reciprocal's leading term refined by one Newton step on the pair
__device__ __forceinline__ double tc_pow_neg_int(double x, int k) {
  double h = x, l = 0.0;
  for (int i = 1; i < k; i++) {
    const double p = h * x;
    const double e = __fma_rn(h, x, -p);
    h = p;
    l = __fma_rn(l, x, e);
    const double s = h + l;
    l = l - (s - h);
    h = s;
  }
  const double y = 1.0 / h;
  // residual of y (h + l) - 1 in extended precision
  const double r = __fma_rn(-y, h, 1.0) - y * l;
  return __fma_rn(y, r, y);
}

struct TcTravCounters {
  unsigned long long frontier[3];  // rotating frontier sizes
  unsigned long long n_m2l, n_p2p;
};

__device__ __forceinline__ unsigned long long tc_warp_append(unsigned long long* counter, bool want) {
  unsigned mask = __ballot_sync(0xffffffffu, want);
  if (!mask) return 0;
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + __popc(mask & ((1u << lane) - 1u));
}

__global__ void k_trav_init(int2* frontier, TcTravCounters* cnt) {
  if (threadIdx.x || blockIdx.x) return;
  frontier[0] = make_int2(0, 0);
  cnt->frontier[0] = 1;
  cnt->frontier[1] = 0;
  cnt->frontier[2] = 0;
  cnt->n_m2l = 0;
  cnt->n_p2p = 0;
}

// step s reads frontier slot s%3, writes slot (s+1)%3 and clears slot (s+2)%3
__global__ void k_trav_step(int s, const int2* __restrict__ fin, int2* __restrict__ fout, unsigned long long fcap,
                            TcTravCounters* cnt, const TcCells c, double theta2, int top_variant, int sbits,
                            unsigned long long* __restrict__ m2l, unsigned long long m2l_cap,
                            unsigned long long* __restrict__ p2p, unsigned long long p2p_cap, unsigned int* err,
                            const TcMac mac = TcMac()) {
  unsigned long long nin = cnt->frontier[s % 3];
  if (nin > fcap) nin = fcap;  // an overflowed step was flagged; never read past the buffer
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt->frontier[(s + 2) % 3] = 0;
  unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long nround = (nin + stride - 1) / stride * stride;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < nround; k += stride) {
    bool valid = k < nin;
    int i = 0, j = 0;
    int act = -1;  // 0 m2l, 1 p2p, 2 split i, 3 split j
    if (valid) {
      int2 pr = fin[k];
      i = pr.x;
      j = pr.y;
      double dx = c.X[i] - c.X[j], dy = c.Y[i] - c.Y[j], dz = c.Z[i] - c.Z[j];
      double rs = c.R[i] + c.R[j];
      int nci = c.nchild[i], ncj = c.nchild[j];
      bool accept;
      if (mac.mode == 0) {
        double R2 = (dx * dx + dy * dy + dz * dz) * theta2;
        accept = R2 > rs * rs;
      } else if (mac.mode == 1) {
        accept = dx * dx + dy * dy + dz * dz > rs * rs * 3;
      } else if (mac.mode == 3) {
        // f2 only, pre-test |d|^2 0.4 > (Ra + Rb)^2; operation order and contractions of the
        // reference's x86-64 build (norm(): fma(dz, dz, fma(dx, dx, dy dy)); Eba += (Pn pa) comb
        // as one fma; R^-(P+1) correctly rounded)
        const double R2 = __fma_rn(dz, dz, __fma_rn(dx, dx, __dmul_rn(dy, dy)));
        double f2 = 10;
        const double Ra = c.R[i], Rb = c.R[j];
        if (__dmul_rn(R2, 0.4) > __dmul_rn(rs, rs)) {
          const int P = mac.p;
          const double Rp = tc_pow_neg_int(__dsqrt_rn(R2), P + 1);
          double pa = 1, Eba = 0;
          for (int k = 0; k <= P; k++) {
            Eba = __fma_rn(__dmul_rn(mac.pn[(size_t)j * (P + 1) + P - k], pa), mac.comb[k], Eba);
            pa = __dmul_rn(pa, Ra);
          }
          const double fac = __dmul_rn(__dmul_rn(8.0, fmax(Ra, Rb)), Rp);
          f2 = __ddiv_rn(__dmul_rn(fac, Eba), __dmul_rn(mac.min_acc[i], mac.fa));
        }
        accept = f2 < 1;
      } else {
        const double R2 = dx * dx + dy * dy + dz * dz;
        double f1 = 10, f2 = 10;
        const double Ra = c.R[i], Rb = c.R[j];
        if (R2 > rs * rs) {
          const double R = sqrt(R2);
          double Rp = R2, pa = 1, pb = 1, Eba = 0, Eab = 0;
          const int P = mac.p;
          for (int k = 0; k <= P; k++) {
            const double fac = mac.comb[k];
            Eab += mac.pn[(size_t)i * (P + 1) + P - k] * pb * fac;
            Eba += mac.pn[(size_t)j * (P + 1) + P - k] * pa * fac;
            pa *= Ra;
            pb *= Rb;
            Rp *= R;
          }
          const double fac = 8 * fmax(Ra, Rb) / rs / Rp;
          Eab *= fac;
          f1 = Eab / (mac.fa * mac.min_acc[j]);
          Eba *= fac;
          f2 = Eba / (mac.fa * mac.min_acc[i]);
        }
        accept = f2 < 1 && f1 < 1;
      }
      if (accept) {
        int ni = c.nbody[i], nj = c.nbody[j];
        act = (mac.mode != 1 && top_variant && ((ni <= 2 && nj <= 8) || (nj <= 2 && ni <= 8))) ? 1 : 0;
        if (mac.p2p_max > 0 && nci == 0 && (long long)ni * nj <= mac.p2p_max) act = 1;
      } else if (nci == 0 && ncj == 0) {
        act = 1;
      } else if (ncj == 0 || (c.R[i] >= c.R[j] && nci != 0)) {
        act = 2;
      } else {
        act = 3;
      }
    }
    unsigned long long key = ((unsigned long long)(unsigned)i << sbits) | (unsigned)j;
    unsigned long long o = tc_warp_append(&cnt->n_m2l, act == 0);
    if (act == 0) {
      if (o < m2l_cap) m2l[o] = key; else tc_set_err(err, TC_EBIT_M2L_CAP);
    }
    o = tc_warp_append(&cnt->n_p2p, act == 1);
    if (act == 1) {
      if (o < p2p_cap) p2p[o] = key; else tc_set_err(err, TC_EBIT_P2P_CAP);
    }
    // children pairs: reserve per thread with one atomic per warp
    int nadd = act == 2 ? c.nchild[i] : act == 3 ? c.nchild[j] : 0;
    int incl = nadd;
    int lane = threadIdx.x & 31;
    for (int d = 1; d < 32; d <<= 1) {
      int v = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += v;
    }
    int total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long base = 0;
    if (lane == 31 && total) base = atomicAdd(&cnt->frontier[(s + 1) % 3], (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 31) + (incl - nadd);
    if (nadd) {
      if (base + nadd > fcap) {
        tc_set_err(err, TC_EBIT_FRONTIER_CAP);
      } else if (act == 2) {
        int c0 = c.child[i];
        for (int q = 0; q < nadd; q++) fout[base + q] = make_int2(c0 + q, j);
      } else {
        int c0 = c.child[j];
        for (int q = 0; q < nadd; q++) fout[base + q] = make_int2(i, c0 + q);
      }
    }
  }
}

// (target << sbits | source) keys, sorted: per-target CSR offsets (targets in [0, ncell))
// (ndev, ncdev optional: counts on the device for device-sized launches; n is then the capacity)
__global__ void k_list_csr(const unsigned long long* __restrict__ keys, unsigned long long n, int ncell, int sbits,
                           int* __restrict__ tgt_start, int* __restrict__ src,
                           const unsigned long long* ndev = nullptr, const int* ncdev = nullptr) {
  if (ndev && *ndev < n) n = *ndev;
  if (ncdev) ncell = *ncdev;
  const unsigned long long smask = (1ull << sbits) - 1ull;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long key = keys[k];
    int t = (int)(key >> sbits);
    src[k] = (int)(key & smask);
    int tp = k == 0 ? -1 : (int)(keys[k - 1] >> sbits);
    for (int q = tp + 1; q <= t; q++) tgt_start[q] = (int)k;
    if (k == n - 1)
      for (int q = t + 1; q <= ncell; q++) tgt_start[q] = (int)n;
  }
  if (n == 0 && blockIdx.x == 0)
    for (int q = threadIdx.x; q <= ncell; q += blockDim.x) tgt_start[q] = 0;
}

// compact list of targets that have at least one entry
__global__ void k_list_targets(const int* __restrict__ tgt_start, int ncell, int* __restrict__ tlist,
                               unsigned int* __restrict__ ntl, const int* ncdev = nullptr) {
  if (ncdev) ncell = *ncdev;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool has = i < ncell && tgt_start[i + 1] > tgt_start[i];
  unsigned mask = __ballot_sync(0xffffffffu, has);
  int lane = threadIdx.x & 31;
  unsigned base = 0;
  if (lane == 0 && mask) base = atomicAdd(ntl, (unsigned)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (has) tlist[base + __popc(mask & ((1u << lane) - 1u))] = i;
}

}  // namespace tc
