// Shared device-side definitions of the B200 FMM gravity evaluation.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/taichi_b200.h"

#define TC_MAX_LEVEL 21          // 63-bit Morton keys carry 21 bits per axis
#define TC_WARP 32
#define TC_NTERM(p) (((p) + 1) * ((p) + 1))
#define TC_PMAX_DEV 16

// device error bits (tc_ctx::d_err)
#define TC_EBIT_M2L_CAP 1u
#define TC_EBIT_P2P_CAP 2u
#define TC_EBIT_FRONTIER_CAP 4u
#define TC_EBIT_DEPTH 8u
#define TC_EBIT_MINIBALL 16u
#define TC_EBIT_NAN 32u
#define TC_EBIT_CELL_CAP 64u
#define TC_EBIT_TIMEOUT 128u

// Sorted-body structure of arrays (Morton order).
struct TcBodies {
  double *x, *y, *z, *m, *vx, *vy, *vz;
  uint8_t* flags;  // bit0 sink, bit1 source
  int* perm;       // sorted position -> caller index
  double eps2 = 0.0;  // Plummer softening squared of the pair interactions (0: Newtonian)
  // mixed near field only: per body (xh yh zh mh) (xl yl zl ml) (vx vy vz 0), FP32 (hi, lo) splits
  // of the position and of the source mass (0 for a non-source), filled by k_body_f32
  float4* f32 = nullptr;
};

// Cells in breadth-first order; level l occupies [lvl_start[l], lvl_start[l+1]).
struct TcCells {
  int *begin, *nbody, *nchild, *child, *parent, *level;
  double *gx, *gy, *gz;        // geometric centre (octree split point)
  double *X, *Y, *Z, *R;       // expansion centre and radius (smallest enclosing ball)
  uint8_t* has_sink;
  double *M, *Md, *L, *Ld;     // ncell x NTERM each (Md/Ld only with jerks)
};

struct TcRootInfo {
  double X0[3];
  double R0;
};

__device__ __forceinline__ void tc_set_err(unsigned int* err, unsigned int bit) { atomicOr(err, bit); }

// exact power-of-two scaling R0 / 2^level as the reference computes R / (1 << level)
__device__ __forceinline__ double tc_level_radius(double R0, int level) { return R0 / (double)(1 << level); }

__device__ __forceinline__ int tc_octant(double x, double y, double z, double cx, double cy, double cz) {
  return (x >= cx) + ((y >= cy) << 1) + ((z >= cz) << 2);
}

// Constant tables, initialised from the host once per device (the library is compiled as a
// single translation unit, so these are the only copies).
__constant__ double c_fact[2 * TC_PMAX_DEV + 2];  // n!
__constant__ double c_tdesign[192];               // 64-point spherical 7-design
