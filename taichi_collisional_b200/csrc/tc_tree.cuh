// Tree build on the device: bounding box, 63-bit Morton keys, LSD radix sort, and the
// level-by-level octree split.  Restates build_tree.h:239-260 (getBounds), :443-454 (Morton
// integers), :459-462 (sort by Body::operator<, exafmm.h:31-40) and :344-435
// (buildCellsSorted): a cell splits when it holds more than ncrit bodies; the split point is
// the cell's geometric centre and the octant test is x >= centre in FP64, found by binary
// search over the Morton-sorted bodies (direct counting for <= 32 bodies).  The reference
// recurses depth first; here each level is split in one launch and cells are stored
// breadth first.
#pragma once
#include "tc_common.cuh"

namespace tc {

constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;

// ---------------------------------------------------------------------------------------
// bounding box (getBounds, build_tree.h:239-260; jerks shift taichi_with_jerks :253-268)
// ---------------------------------------------------------------------------------------
__global__ void k_bounds_partial(int n, const double* __restrict__ x, const double* __restrict__ y,
                                 const double* __restrict__ z, const double* __restrict__ m,
                                 double* __restrict__ part, unsigned int* err) {
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double a = x[i], b = y[i], c = z[i], w = m[i];
    bad |= !(isfinite(a) && isfinite(b) && isfinite(c) && isfinite(w));
    mn[0] = fmin(mn[0], a); mx[0] = fmax(mx[0], a);
    mn[1] = fmin(mn[1], b); mx[1] = fmax(mx[1], b);
    mn[2] = fmin(mn[2], c); mx[2] = fmax(mx[2], c);
  }
  if (bad) tc_set_err(err, TC_EBIT_NAN);
  for (int o = 16; o > 0; o >>= 1)
    for (int d = 0; d < 3; d++) {
      mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
  __shared__ double s[32][6];
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
    for (int d = 0; d < 3; d++) { s[w][d] = mn[d]; s[w][3 + d] = mx[d]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); k++)
      for (int d = 0; d < 3; d++) { s[0][d] = fmin(s[0][d], s[k][d]); s[0][3 + d] = fmax(s[0][3 + d], s[k][3 + d]); }
    for (int d = 0; d < 6; d++) part[6 * blockIdx.x + d] = s[0][d];
  }
}

__global__ void k_bounds_final(int nblk, const double* __restrict__ part, TcRootInfo* root, int use_shift,
                               double u0, double u1, double u2) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int b = 0; b < nblk; b++)
    for (int d = 0; d < 3; d++) { mn[d] = fmin(mn[d], part[6 * b + d]); mx[d] = fmax(mx[d], part[6 * b + 3 + d]); }
  double X0[3], R0 = 0;
  for (int d = 0; d < 3; d++) X0[d] = __ddiv_rn(__dadd_rn(mx[d], mn[d]), 2.0);
  if (use_shift) {
    double box = -1, u[3] = {u0, u1, u2};
    for (int d = 0; d < 3; d++) if (__dsub_rn(mx[d], mn[d]) > box) box = __dsub_rn(mx[d], mn[d]);
    for (int d = 0; d < 3; d++) X0[d] = __dadd_rn(X0[d], __ddiv_rn(__dmul_rn(__dsub_rn(u[d], 0.5), box), 25.0));
  }
  for (int d = 0; d < 3; d++) {
    R0 = fmax(__dsub_rn(X0[d], mn[d]), R0);
    R0 = fmax(__dsub_rn(mx[d], X0[d]), R0);
  }
  R0 = __dmul_rn(R0, 1.00001);
  for (int d = 0; d < 3; d++) root->X0[d] = X0[d];
  root->R0 = R0;
}

// ---------------------------------------------------------------------------------------
// Morton keys: the reference's 28-bit integers floor((x - (X0 - R0)) / (2 R0) * 2^28)
// (build_tree.h:448-453), truncated to their top 21 bits and interleaved with z as the most
// significant bit of each triple (the order Body::operator< defines, exafmm.h:31-40).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long tc_spread21(unsigned long long v) {
  v &= 0x1fffffull;
  v = (v | v << 32) & 0x1f00000000ffffull;
  v = (v | v << 16) & 0x1f0000ff0000ffull;
  v = (v | v << 8) & 0x100f00f00f00f00full;
  v = (v | v << 4) & 0x10c30c30c30c30c3ull;
  v = (v | v << 2) & 0x1249249249249249ull;
  return v;
}

__device__ __forceinline__ uint32_t tc_morton28(double x, double lo, double twoR0) {
  double f = __ddiv_rn(__dsub_rn(x, lo), twoR0);
  return (uint32_t)(long long)floor(__dmul_rn(f, 268435456.0));
}

__global__ void k_morton(int n, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, const TcRootInfo* __restrict__ root,
                         unsigned long long* __restrict__ key, int* __restrict__ val) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double R0 = root->R0, two = __dmul_rn(2.0, R0);
  uint32_t ix = tc_morton28(x[i], __dsub_rn(root->X0[0], R0), two);
  uint32_t iy = tc_morton28(y[i], __dsub_rn(root->X0[1], R0), two);
  uint32_t iz = tc_morton28(z[i], __dsub_rn(root->X0[2], R0), two);
  key[i] = tc_spread21(ix >> 7) | (tc_spread21(iy >> 7) << 1) | (tc_spread21(iz >> 7) << 2);
  val[i] = i;
}

// ---------------------------------------------------------------------------------------
// Stable LSD radix sort, 8 bits per pass: per-tile digit histograms, one exclusive scan in
// (digit, tile) order, then a stable scatter (ranks from warp match + per-warp counts).
// ---------------------------------------------------------------------------------------
// ndev (optional): the key count on the device (device-sized launches); n is then the capacity
__global__ void k_rs_hist(const unsigned long long* __restrict__ keys, int n, int shift, uint32_t* __restrict__ hist,
                          const unsigned long long* ndev = nullptr) {
  __shared__ uint32_t h[256];
  if (ndev && *ndev < (unsigned long long)n) n = (int)*ndev;
  int t = threadIdx.x;
  int base = blockIdx.x * kRsTile;
  if (base >= n) {  // a tile past the keys (device-sized launch): an empty histogram
    hist[t * gridDim.x + blockIdx.x] = 0u;
    return;
  }
  h[t] = 0;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRsItems; r++) {
    int idx = base + r * kRsThreads + t;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[t * gridDim.x + blockIdx.x] = h[t];
}

// single-block exclusive scan (in place) of `total` counters
__global__ void k_excl_scan_u32(uint32_t* __restrict__ a, int total, uint32_t* __restrict__ sum_out) {
  __shared__ uint32_t s[1024];
  int t = threadIdx.x, T = blockDim.x;
  int chunk = (total + T - 1) / T;
  int b = t * chunk, e = min(total, b + chunk);
  uint32_t loc = 0;
  for (int i = b; i < e; i++) loc += a[i];
  s[t] = loc;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    uint32_t v = t >= o ? s[t - o] : 0u;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  uint32_t run = s[t] - loc;
  for (int i = b; i < e; i++) {
    uint32_t v = a[i];
    a[i] = run;
    run += v;
  }
  if (t == T - 1 && sum_out) *sum_out = s[t];
}

// multi-block exclusive scan: 4096 counters per block, then the block sums, then the fix-up
constexpr int kScanThreads = 1024, kScanItems = 4;
__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(uint32_t* __restrict__ a, int total,
                                                              uint32_t* __restrict__ sums) {
  __shared__ uint32_t s[kScanThreads];
  int t = threadIdx.x;
  int base = blockIdx.x * kScanThreads * kScanItems + t * kScanItems;
  uint32_t v[kScanItems], loc = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    v[i] = base + i < total ? a[base + i] : 0u;
    loc += v[i];
  }
  s[t] = loc;
  __syncthreads();
  for (int o = 1; o < kScanThreads; o <<= 1) {
    uint32_t w = t >= o ? s[t - o] : 0u;
    __syncthreads();
    s[t] += w;
    __syncthreads();
  }
  uint32_t run = s[t] - loc;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    if (base + i < total) a[base + i] = run;
    run += v[i];
  }
  if (t == kScanThreads - 1) sums[blockIdx.x] = s[t];
}

__global__ void k_scan_add(uint32_t* __restrict__ a, int total, const uint32_t* __restrict__ sums) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) a[i] += sums[i / (kScanThreads * kScanItems)];
}

// exclusive scan of a[total] in place; sums needs total / 4096 + 1 entries
inline int excl_scan(uint32_t* a, int total, uint32_t* sums, cudaStream_t st) {
  int nb = (total + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
  if (nb <= 1) {
    k_excl_scan_u32<<<1, 1024, 0, st>>>(a, total, nullptr);
    return 1;
  }
  k_scan_blocks<<<nb, kScanThreads, 0, st>>>(a, total, sums);
  k_excl_scan_u32<<<1, 1024, 0, st>>>(sums, nb, nullptr);
  k_scan_add<<<(total + 255) / 256, 256, 0, st>>>(a, total, sums);
  return 3;
}

template <bool kVals>
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const unsigned long long* __restrict__ kin, const int* __restrict__ vin,
                                                           unsigned long long* __restrict__ kout, int* __restrict__ vout, int n,
                                                           int shift, const uint32_t* __restrict__ hist,
                                                           const unsigned long long* ndev = nullptr) {
  __shared__ uint32_t s_base[256];
  if (ndev && *ndev < (unsigned long long)n) n = (int)*ndev;
  if ((long long)blockIdx.x * kRsTile >= n) return;  // a tile past the keys: nothing to move
  __shared__ uint32_t s_wcnt[kRsThreads / 32][257];
  int t = threadIdx.x, w = t >> 5, lane = t & 31;
  s_base[t] = hist[t * gridDim.x + blockIdx.x];
  unsigned lt = (1u << lane) - 1u;
  int base = blockIdx.x * kRsTile;
  for (int r = 0; r < kRsItems; r++) {
    for (int k = lane; k < 257; k += 32) s_wcnt[w][k] = 0;
    __syncthreads();
    int idx = base + r * kRsThreads + t;
    bool valid = idx < n;
    unsigned long long key = valid ? kin[idx] : 0ull;
    int digit = valid ? (int)((key >> shift) & 255u) : 256;
    unsigned peers = __match_any_sync(0xffffffffu, digit);
    int rank = __popc(peers & lt);
    if (lane == __ffs(peers) - 1) s_wcnt[w][digit] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t off = s_base[digit] + rank;
      for (int k = 0; k < w; k++) off += s_wcnt[k][digit];
      kout[off] = key;
      if (kVals) vout[off] = vin[idx];
    }
    __syncthreads();
    uint32_t tot = 0;
    for (int k = 0; k < kRsThreads / 32; k++) tot += s_wcnt[k][t];
    s_base[t] += tot;
    __syncthreads();
  }
}

// Sorts (keys, vals) by key bits [0, bits).  Uses alt buffers; the result ends in keys/vals.
// Device-sized form (ndev given, n = capacity): no copy back; *kfinal receives the buffer that
// holds the sorted keys.
inline int radix_sort(unsigned long long* keys, int* vals, unsigned long long* keys_alt, int* vals_alt, int n, int bits, uint32_t* hist,
                      cudaStream_t st, int begin_bit = 0, const unsigned long long* ndev = nullptr,
                      unsigned long long** kfinal = nullptr) {
  if (kfinal) *kfinal = keys;
  if (n <= 1 && !ndev) return 0;
  int launches = 0;
  int nblk = (n + kRsTile - 1) / kRsTile;
  int passes = (bits - begin_bit + 7) / 8;
  unsigned long long *ka = keys, *kb = keys_alt;
  int *va = vals, *vb = vals_alt;
  for (int p = 0; p < passes; p++) {
    int shift = begin_bit + 8 * p;
    k_rs_hist<<<nblk, kRsThreads, 0, st>>>(ka, n, shift, hist, ndev);
    launches += 2 + excl_scan(hist, 256 * nblk, hist + 256 * (size_t)nblk, st);
    if (vals)
      k_rs_scatter<true><<<nblk, kRsThreads, 0, st>>>(ka, va, kb, vb, n, shift, hist, ndev);
    else
      k_rs_scatter<false><<<nblk, kRsThreads, 0, st>>>(ka, nullptr, kb, nullptr, n, shift, hist, ndev);
    unsigned long long* tk = ka; ka = kb; kb = tk;
    int* tv = va; va = vb; vb = tv;
  }
  if (kfinal) {
    *kfinal = ka;
    return launches;
  }
  if (ka != keys) {
    cudaMemcpyAsync(keys, ka, sizeof(unsigned long long) * n, cudaMemcpyDeviceToDevice, st);
    if (vals) cudaMemcpyAsync(vals, va, sizeof(int) * n, cudaMemcpyDeviceToDevice, st);
  }
  return launches;
}

// gather the caller's arrays into Morton order
__global__ void k_gather_bodies(int n, const int* __restrict__ perm, const double* __restrict__ x,
                                const double* __restrict__ y, const double* __restrict__ z,
                                const double* __restrict__ m, const double* __restrict__ vx,
                                const double* __restrict__ vy, const double* __restrict__ vz,
                                const uint8_t* __restrict__ flags, TcBodies b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int j = perm[i];
  b.perm[i] = j;
  b.x[i] = x[j]; b.y[i] = y[j]; b.z[i] = z[j]; b.m[i] = m[j];
  if (b.vx) {
    b.vx[i] = vx ? vx[j] : 0.0; b.vy[i] = vy ? vy[j] : 0.0; b.vz[i] = vz ? vz[j] : 0.0;
  }
  b.flags[i] = flags ? (flags[j] & 3u) : 3u;
}

// ---------------------------------------------------------------------------------------
// Octree levels
// ---------------------------------------------------------------------------------------
struct TcLevels {
  int start[TC_MAX_LEVEL + 3];
  int count[TC_MAX_LEVEL + 3];
  int ncell;
};

__global__ void k_tree_root(int n, TcCells c, const TcRootInfo* root, TcLevels* lv) {
  if (threadIdx.x || blockIdx.x) return;
  c.begin[0] = 0; c.nbody[0] = n; c.nchild[0] = 0; c.child[0] = -1; c.parent[0] = -1; c.level[0] = 0;
  c.gx[0] = root->X0[0]; c.gy[0] = root->X0[1]; c.gz[0] = root->X0[2];
  for (int l = 0; l < TC_MAX_LEVEL + 3; l++) { lv->start[l] = 0; lv->count[l] = 0; }
  lv->start[0] = 0; lv->count[0] = 1; lv->start[1] = 1; lv->ncell = 1;
}

// decide splits of the cells of level l; off[8*k + o] = first body of octant o
__global__ void k_tree_split(int l, int ncrit, const TcBodies b, TcCells c, const TcLevels* lv, int* __restrict__ off,
                             unsigned int* err) {
  int cnt = lv->count[l], st = lv->start[l];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    int ci = st + k;
    int beg = c.begin[ci], nb = c.nbody[ci], end = beg + nb;
    double X = c.gx[ci], Y = c.gy[ci], Z = c.gz[ci];
    if (nb <= ncrit) { c.nchild[ci] = 0; continue; }
    if (l >= TC_MAX_LEVEL) { c.nchild[ci] = 0; tc_set_err(err, TC_EBIT_DEPTH); continue; }
    int o8[9];
    if (nb <= 32) {
      int size[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int i = beg; i < end; i++) size[tc_octant(b.x[i], b.y[i], b.z[i], X, Y, Z)]++;
      int o = beg;
      for (int q = 0; q < 8; q++) { o8[q] = o; o += size[q]; }
    } else {
      o8[0] = beg;
      for (int q = 1; q < 8; q++) {
        int left = beg, right = end;
        while (left < right - 1) {
          int mid = (left + right) / 2;
          if (tc_octant(b.x[mid], b.y[mid], b.z[mid], X, Y, Z) >= q) right = mid; else left = mid;
        }
        o8[q] = left + 1;
      }
    }
    o8[8] = end;
    int nch = 0;
    for (int q = 0; q < 8; q++) {
      off[8 * k + q] = o8[q];
      nch += (q < 7 ? o8[q + 1] : end) - o8[q] > 0;
    }
    c.nchild[ci] = nch;
  }
}

// exclusive scan of nchild over level l (single block) -> child indices, level l+1 range
__global__ void k_tree_scan(int l, TcCells c, TcLevels* lv, int cell_cap, unsigned int* err) {
  __shared__ int s[1024];
  int cnt = lv->count[l], st = lv->start[l];
  int t = threadIdx.x, T = blockDim.x;
  int chunk = (cnt + T - 1) / T;
  int b = t * chunk, e = min(cnt, b + chunk);
  int loc = 0;
  for (int i = b; i < e; i++) loc += c.nchild[st + i];
  s[t] = loc;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    int v = t >= o ? s[t - o] : 0;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  int next = st + cnt;
  int run = s[t] - loc;
  // over capacity: the level's cells stay leaves, so the (flagged) tree remains consistent for
  // launches that follow without a host check (a captured graph)
  const bool over = next + s[T - 1] > cell_cap;
  for (int i = b; i < e; i++) {
    int nc = c.nchild[st + i];
    if (over) {
      c.nchild[st + i] = 0;
      c.child[st + i] = -1;
      continue;
    }
    c.child[st + i] = nc ? next + run : -1;
    run += nc;
  }
  if (t == T - 1) {
    int total = s[t];
    if (over) {
      tc_set_err(err, TC_EBIT_CELL_CAP);
      total = 0;
    }
    lv->count[l + 1] = total;
    lv->start[l + 1] = next;
    lv->start[l + 2] = next + total;
    lv->ncell = next + total;
  }
}

__global__ void k_tree_emit(int l, TcCells c, const TcLevels* lv, const int* __restrict__ off,
                            const TcRootInfo* root) {
  int cnt = lv->count[l], st = lv->start[l];
  if (lv->count[l + 1] == 0) return;
  double r = tc_level_radius(root->R0, l + 1);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    int ci = st + k;
    if (c.nchild[ci] == 0) continue;
    int end = c.begin[ci] + c.nbody[ci];
    int ch = c.child[ci];
    for (int q = 0; q < 8; q++) {
      int b0 = off[8 * k + q], b1 = q < 7 ? off[8 * k + q + 1] : end;
      if (b1 <= b0) continue;
      c.begin[ch] = b0; c.nbody[ch] = b1 - b0; c.nchild[ch] = 0; c.child[ch] = -1; c.parent[ch] = ci;
      c.level[ch] = l + 1;
      c.gx[ch] = __dadd_rn(c.gx[ci], (q & 1) ? r : -r);
      c.gy[ch] = __dadd_rn(c.gy[ci], (q & 2) ? r : -r);
      c.gz[ch] = __dadd_rn(c.gz[ci], (q & 4) ? r : -r);
      ch++;
    }
  }
}

}  // namespace tc
