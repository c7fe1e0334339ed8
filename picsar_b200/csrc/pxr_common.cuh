// Shared device helpers for the picsar_b200 CUDA kernels (sm_100a).
//
// Index conventions follow PICSAR's Fortran arrays: a guarded grid has
// lower bound -g and upper bound n+g per axis, column-major (x fastest); the
// base pointer addresses element (-gx,-gy,-gz).  Shape-factor formulas are
// those of src/particle_pushers/particle_pusher_manager_3d.F90:1287-2193
// (gather) and src/particle_deposition/current_deposition/esirkepov/
// esirkepov_3d.F90 (deposition).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

// The status codes (PXRB_OK, PXRB_EINVAL, ...) returned by every extern "C"
// entry point are defined once, in the public header.
#include "picsar_b200.h"

typedef int64_t i64;

#define PXRB_CHECK_LAUNCH()                                  \
  do {                                                       \
    cudaError_t e_ = cudaGetLastError();                     \
    if (e_ != cudaSuccess) return PXRB_ELAUNCH;              \
  } while (0)

// Guarded column-major grid descriptor.
struct GridG {
  i64 nx, ny, nz;     // cells (nodes 0..n)
  i64 gx, gy, gz;     // guards
  i64 sx, sy;         // strides of y and z: sx = NX, sy = NX*NY
  __host__ __device__ inline i64 idx(i64 i, i64 j, i64 k) const {
    return (i + gx) + sx * (j + gy) + sy * (k + gz);
  }
  __host__ __device__ inline i64 size() const { return sy * (nz + 1 + 2 * gz); }
};

inline GridG make_grid(i64 nx, i64 ny, i64 nz, i64 gx, i64 gy, i64 gz) {
  GridG g;
  g.nx = nx; g.ny = ny; g.nz = nz; g.gx = gx; g.gy = gy; g.gz = gz;
  g.sx = nx + 1 + 2 * gx;
  g.sy = g.sx * (ny + 1 + 2 * gy);
  return g;
}

// Fortran FLOOR and NINT (round half away from zero) to int.
template <typename R> __device__ __forceinline__ int ffloor(R x) { return (int)floor(x); }
template <> __device__ __forceinline__ int ffloor<float>(float x) { return (int)floorf(x); }
template <typename R> __device__ __forceinline__ int fnint(R x) { return (int)round(x); }
template <> __device__ __forceinline__ int fnint<float>(float x) { return (int)roundf(x); }

// ---------------------------------------------------------------------------
// Shape factors.  N = number of support points; the first point sits at
// index i0.  Node-centred ("full") shapes of order 1..3 and the
// staggered shapes of the energy-conserving gather with
// l_lower_order_in_v = .TRUE. (order-1 lower, at the index the fused Fortran
// kernels use).
// ---------------------------------------------------------------------------
template <int ORDER, typename R> struct NodeShape {
  static constexpr int N = ORDER + 1;
  int i0;
  R s[N];
  __device__ __forceinline__ void set(R x) {
    if (ORDER == 1) {
      int j = ffloor(x);
      R xi = x - (R)j;
      i0 = j; s[0] = (R)1 - xi; s[1] = xi;
    } else if (ORDER == 2) {
      int j = fnint(x);
      R xi = x - (R)j, xs = xi * xi;
      i0 = j - 1;
      s[0] = (R)0.5 * ((R)0.5 - xi) * ((R)0.5 - xi);
      s[1] = (R)0.75 - xs;
      s[2] = (R)0.5 * ((R)0.5 + xi) * ((R)0.5 + xi);
    } else {
      int j = ffloor(x);
      R xi = x - (R)j, ox = (R)1 - xi, xs = xi * xi, oxs = ox * ox;
      i0 = j - 1;
      s[0] = (R)(1.0 / 6.0) * oxs * ox;
      s[1] = (R)(2.0 / 3.0) - xs * ((R)1 - xi * (R)0.5);
      s[2] = (R)(2.0 / 3.0) - oxs * ((R)1 - ox * (R)0.5);
      s[3] = (R)(1.0 / 6.0) * xs * xi;
    }
  }
};

template <int ORDER, typename R> struct StagShape {
  static constexpr int N = ORDER;  // one order lower
  int i0;
  R s[N > 0 ? N : 1];
  __device__ __forceinline__ void set(R x) {
    if (ORDER == 1) {
      i0 = ffloor(x); s[0] = (R)1;
    } else if (ORDER == 2) {
      int j0 = ffloor(x - (R)0.5);
      R xi = x - (R)0.5 - (R)j0;
      i0 = j0; s[0] = (R)1 - xi; s[1] = xi;
    } else {
      int j0 = ffloor(x);
      R xi = x - (R)0.5 - (R)j0, xs = xi * xi;
      i0 = j0 - 1;
      s[0] = (R)0.5 * ((R)0.5 - xi) * ((R)0.5 - xi);
      s[1] = (R)0.75 - xs;
      s[2] = (R)0.5 * ((R)0.5 + xi) * ((R)0.5 + xi);
    }
  }
};

// ---------------------------------------------------------------------------
// Momentum pushers (per particle).
// Boris: src/particle_pushers/boris_pusher/boris_3d.F90:96-131, followed by
// pxr_set_gamma (:1092-1099).  Vay (which = 0): vay_pusher/vay_3d.F90:100-130.
// ---------------------------------------------------------------------------
// 1/sqrt(x) and a/b: correctly rounded in FP64; in FP32 the hardware
// approximations (rsqrtf, __fdividef: a few ulp), well inside the FP32
// engine's error budget and several instructions shorter each.
template <typename R> __device__ __forceinline__ R inv_sqrt(R x) { return (R)1 / sqrt(x); }
template <> __device__ __forceinline__ float inv_sqrt<float>(float x) { return rsqrtf(x); }
template <typename R> __device__ __forceinline__ R quot(R a, R b) { return a / b; }
template <> __device__ __forceinline__ float quot<float>(float a, float b) { return __fdividef(a, b); }

template <typename R>
__device__ __forceinline__ void boris_push(R& ux, R& uy, R& uz, R& gi, R ex, R ey, R ez,
                                           R bx, R by, R bz, R cst, R clghtisq) {
  ux = ux + ex * cst; uy = uy + ey * cst; uz = uz + ez * cst;
  R usq = (ux * ux + uy * uy + uz * uz) * clghtisq;
  R gt = inv_sqrt<R>((R)1 + usq);
  R tx = gt * bx * cst, ty = gt * by * cst, tz = gt * bz * cst;
  R tsqi = quot<R>((R)2, (R)1 + tx * tx + ty * ty + tz * tz);
  R sx = tx * tsqi, sy = ty * tsqi, sz = tz * tsqi;
  R uxp = ux + uy * tz - uz * ty;
  R uyp = uy + uz * tx - ux * tz;
  R uzp = uz + ux * ty - uy * tx;
  ux = ux + uyp * sz - uzp * sy;
  uy = uy + uzp * sx - uxp * sz;
  uz = uz + uxp * sy - uyp * sx;
  ux = ux + ex * cst; uy = uy + ey * cst; uz = uz + ez * cst;
  usq = (ux * ux + uy * uy + uz * uz) * clghtisq;
  gi = inv_sqrt<R>((R)1 + usq);
}

template <typename R>
__device__ __forceinline__ void set_gamma(R ux, R uy, R uz, R& gi, R clghtisq) {
  R usq = (ux * ux + uy * uy + uz * uz) * clghtisq;
  gi = inv_sqrt<R>((R)1 + usq);
}

// which = 0 full Vay push; const = q dt / m.
template <typename R>
__device__ __forceinline__ void vay_push(R& ux, R& uy, R& uz, R& gi, R ex, R ey, R ez, R bx,
                                         R by, R bz, R cst, R invclight, R invclightsq) {
  R bconst = (R)0.5 * cst;
  R taux = bconst * bx, tauy = bconst * by, tauz = bconst * bz;
  R tausq = taux * taux + tauy * tauy + tauz * tauz;
  R uxpr = ux + cst * ex + (uy * tauz - uz * tauy) * gi;
  R uypr = uy + cst * ey + (uz * taux - ux * tauz) * gi;
  R uzpr = uz + cst * ez + (ux * tauy - uy * taux) * gi;
  R gprsq = ((R)1 + (uxpr * uxpr + uypr * uypr + uzpr * uzpr) * invclightsq);
  R ust = (uxpr * taux + uypr * tauy + uzpr * tauz) * invclight;
  R sigma = gprsq - tausq;
  R gisq = quot<R>((R)2, sigma + sqrt(sigma * sigma + (R)4 * (tausq + ust * ust)));
  gi = sqrt(gisq);
  R bg = bconst * gi;
  R tx = bg * bx, ty = bg * by, tz = bg * bz;
  R s = quot<R>((R)1, (R)1 + tausq * gisq);
  R tu = tx * uxpr + ty * uypr + tz * uzpr;
  ux = s * (uxpr + tx * tu + uypr * tz - uzpr * ty);
  uy = s * (uypr + ty * tu + uzpr * tx - uxpr * tz);
  uz = s * (uzpr + tz * tu + uxpr * ty - uypr * tx);
}

// ---------------------------------------------------------------------------
// One axis of the Esirkepov box.  The reference evaluates the shape at the
// new position (sx0) and at the old position (sx), shifted by the node
// difference d = node(old) - node(new), and sweeps the box
// [min(0,d) - a, max(0,d) + b] with a = ORDER/2, b = (ORDER+1)/2
// (esirkepov_3d.F90:168-198, :1870-1876, :3413-3418).  Here both shapes are
// stored in box coordinates r = i - box_min (0..ORDER+1) so that every index
// is a compile-time constant.  |d| <= 1 always holds under the CFL limit
// (c dt / dx < 1); `bad` is set otherwise.
// ---------------------------------------------------------------------------
template <int ORDER, typename R> struct EsirAxis {
  static constexpr int M = ORDER + 2;   // maximal box size
  int i0;        // global index of box start
  int n;         // box size: ORDER + 1 + |d|
  R s0[M];       // new-position shape in box coordinates
  R s1[M];       // old-position shape in box coordinates

  // node index and in-cell variable of order ORDER at position x
  __device__ __forceinline__ static int node(R x) {
    return (ORDER == 2) ? fnint(x) : ffloor(x);
  }
  __device__ __forceinline__ static void shape(R xi, R* s) {
    if (ORDER == 1) {
      s[0] = (R)1 - xi; s[1] = xi;
    } else if (ORDER == 2) {
      R xs = xi * xi;
      s[0] = (R)0.5 * ((R)0.5 - xi) * ((R)0.5 - xi);
      s[1] = (R)0.75 - xs;
      s[2] = (R)0.5 * ((R)0.5 + xi) * ((R)0.5 + xi);
    } else {
      R ox = (R)1 - xi, xs = xi * xi, oxs = ox * ox;
      s[0] = (R)(1.0 / 6.0) * oxs * ox;
      s[1] = (R)(2.0 / 3.0) - xs * ((R)1 - xi / (R)2);
      s[2] = (R)(2.0 / 3.0) - oxs * ((R)1 - ox / (R)2);
      s[3] = (R)(1.0 / 6.0) * xs * xi;
    }
  }
  // Build from node indices and in-cell variables of new (n0, xi0) and
  // old (n1, xi1) positions.
  __device__ __forceinline__ bool set(int n0, R xi0, int n1, R xi1) {
    constexpr int a = ORDER / 2;
    int d = n1 - n0;
    bool bad = (d < -1) || (d > 1);
    d = bad ? 0 : d;
    int sh0 = d < 0 ? 1 : 0;   // offset of the new shape in the box
    int sh1 = d > 0 ? 1 : 0;   // offset of the old shape in the box
    i0 = n0 - a - sh0;
    n = ORDER + 1 + (d != 0 ? 1 : 0);
    R t0[ORDER + 1], t1[ORDER + 1];
    shape(xi0, t0);
    shape(xi1, t1);
#pragma unroll
    for (int r = 0; r < M; ++r) {
      R a0 = (r <= ORDER) ? t0[r < ORDER + 1 ? r : ORDER] : (R)0;
      R b0 = (r >= 1) ? t0[r >= 1 ? r - 1 : 0] : (R)0;
      s0[r] = sh0 ? b0 : a0;
      R a1 = (r <= ORDER) ? t1[r < ORDER + 1 ? r : ORDER] : (R)0;
      R b1 = (r >= 1) ? t1[r >= 1 ? r - 1 : 0] : (R)0;
      s1[r] = sh1 ? b1 : a1;
    }
    return !bad;
  }
};
