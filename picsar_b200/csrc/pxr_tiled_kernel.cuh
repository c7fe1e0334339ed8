// Device code of the tiled engine's fused particle kernel (included by the
// per-order translation units pxr_tiled_o{1,2,3}.cu).
#pragma once
#include "pxr_common.cuh"
#include "picsar_b200.h"

namespace pxrt {

typedef pxrb_tiled_job Job;

// ---------------------------------------------------------------------------
// packed cell index: x | y << 11 | z << 22
// ---------------------------------------------------------------------------
__device__ __forceinline__ void unpack_cell(uint32_t c, int& i, int& j, int& k) {
  i = (int)(c & 2047u);
  j = (int)((c >> 11) & 2047u);
  k = (int)(c >> 22);
}
__device__ __forceinline__ uint32_t pack_cell(int i, int j, int k) {
  return (uint32_t)i | ((uint32_t)j << 11) | ((uint32_t)k << 22);
}

// Reach of the gather and deposition stencils around a particle's cell c:
// nodes [c - L, c + H] (also covers the Esirkepov box when the cell changes
// by one, which is accounted for by the window margin).
template <int ORDER> struct Reach {
  static constexpr int L = ORDER == 1 ? 0 : 1;
  static constexpr int H = ORDER == 1 ? 1 : 2;
};

// Row and plane pitch (elements) of a tile's shared-memory window of edge W
// for cubic tiles of edge T.  Padded so that the T^3 cells of the tile fall
// into the 32 bank classes (address mod 32) exactly T^3/32 times each: the
// sort lays out each warp's particles in distinct classes, and equal class
// sizes let it do so for all but the tail of a tile.  Entries: smallest
// window with that property, SY >= W, SZ >= SY * W.
__host__ __device__ constexpr int win_sy(int T, int W) {
  return T == 4 ? (W == 5 ? 6 : W == 7 ? 8 : W == 9 ? 10 : W) : W;
}
__host__ __device__ constexpr int win_sz(int T, int W) {
  return T == 8 ? (W == 9 ? 84 : W == 11 ? 124 : W == 13 ? 172 : W == 15 ? 228 : W * W)
       : T == 4 ? (W == 5 ? 40 : W == 7 ? 58 : W == 9 ? 104 : W * W)
       : W * W;
}

// ---------------------------------------------------------------------------
// Shapes from (cell, offset): x = c + o with o in [0,1).  r0 is the first
// support node relative to c.  Same formulas as NodeShape/StagShape, with
// floor(x) = c and nint(x) = c + (o >= 1/2) for x >= 0.
// ---------------------------------------------------------------------------
template <int ORDER, typename R> struct NodeCO {
  static constexpr int N = ORDER + 1;
  int r0;
  R s[N];
  __device__ __forceinline__ void set(R o) {
    if (ORDER == 1) {
      r0 = 0; s[0] = (R)1 - o; s[1] = o;
    } else if (ORDER == 2) {
      int r = o >= (R)0.5 ? 1 : 0;
      R xi = o - (R)r, xs = xi * xi;
      r0 = r - 1;
      s[0] = (R)0.5 * ((R)0.5 - xi) * ((R)0.5 - xi);
      s[1] = (R)0.75 - xs;
      s[2] = (R)0.5 * ((R)0.5 + xi) * ((R)0.5 + xi);
    } else {
      R xi = o, ox = (R)1 - xi, xs = xi * xi, oxs = ox * ox;
      r0 = -1;
      s[0] = (R)(1.0 / 6.0) * oxs * ox;
      s[1] = (R)(2.0 / 3.0) - xs * ((R)1 - xi * (R)0.5);
      s[2] = (R)(2.0 / 3.0) - oxs * ((R)1 - ox * (R)0.5);
      s[3] = (R)(1.0 / 6.0) * xs * xi;
    }
  }
};

template <int ORDER, typename R> struct StagCO {
  static constexpr int N = ORDER;
  int r0;
  R s[N];
  __device__ __forceinline__ void set(R o) {
    if (ORDER == 1) {
      r0 = 0; s[0] = (R)1;
    } else if (ORDER == 2) {
      int j0 = o >= (R)0.5 ? 0 : -1;
      R xi = o - (R)0.5 - (R)j0;
      r0 = j0; s[0] = (R)1 - xi; s[1] = xi;
    } else {
      R xi = o - (R)0.5, xs = xi * xi;
      r0 = -1;
      s[0] = (R)0.5 * ((R)0.5 - xi) * ((R)0.5 - xi);
      s[1] = (R)0.75 - xs;
      s[2] = (R)0.5 * ((R)0.5 + xi) * ((R)0.5 + xi);
    }
  }
};

// Esirkepov node index (relative to c) and in-cell variable of a position
template <int ORDER, typename R>
__device__ __forceinline__ void esir_node(R o, int& r, R& xi) {
  if (ORDER == 2) {
    r = o >= (R)0.5 ? 1 : 0;
    xi = o - (R)r;
  } else {
    r = 0;
    xi = o;
  }
}

// Field accessor: either a shared-memory window or the global guarded arrays.
template <typename R> struct FieldView {
  const R* p;       // element (0,0,0) of the view
  int sy, sz;       // strides
  __device__ __forceinline__ R at(int i, int j, int k) const { return p[i + sy * j + sz * k]; }
};

template <int NA, int NB, int NC, typename R>
__device__ __forceinline__ R gsum(const FieldView<R>& f, int ia, const R* sa, int ib,
                                  const R* sb, int ic, const R* sc) {
  R out = (R)0;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    R a = (R)0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      R r = (R)0;
#pragma unroll
      for (int t = 0; t < NA; ++t) r = r + sa[t] * f.at(ia + t, ib + b, ic + c);
      a = a + r * sb[b];
    }
    out = out + a * sc[c];
  }
  return out;
}

// Gather E and B at a particle whose cell is (ci, cj, ck) in the view's
// coordinates.
template <int ORDER, typename R>
__device__ __forceinline__ void gather6(const FieldView<R>* F, int ci, int cj, int ck, R ox,
                                        R oy, R oz, R* eb) {
  NodeCO<ORDER, R> nx, ny, nz;
  StagCO<ORDER, R> sx, sy, sz;
  nx.set(ox); ny.set(oy); nz.set(oz);
  sx.set(ox); sy.set(oy); sz.set(oz);
  constexpr int N = ORDER + 1, S = ORDER;
  eb[0] = gsum<S, N, N>(F[0], ci + sx.r0, sx.s, cj + ny.r0, ny.s, ck + nz.r0, nz.s);
  eb[1] = gsum<N, S, N>(F[1], ci + nx.r0, nx.s, cj + sy.r0, sy.s, ck + nz.r0, nz.s);
  eb[2] = gsum<N, N, S>(F[2], ci + nx.r0, nx.s, cj + ny.r0, ny.s, ck + sz.r0, sz.s);
  eb[3] = gsum<N, S, S>(F[3], ci + nx.r0, nx.s, cj + sy.r0, sy.s, ck + sz.r0, sz.s);
  eb[4] = gsum<S, N, S>(F[4], ci + sx.r0, sx.s, cj + ny.r0, ny.s, ck + sz.r0, sz.s);
  eb[5] = gsum<S, S, N>(F[5], ci + sx.r0, sx.s, cj + sy.r0, sy.s, ck + nz.r0, nz.s);
}

// Accumulator target for the deposition: shared window (atomicAdd on A) or
// the global periodic FP64 grid.
template <typename A> struct SmemAcc {
  A* p;
  int sy, sz;
  __device__ __forceinline__ void add(int i, int j, int k, A v) const {
    atomicAdd(p + i + sy * j + sz * k, v);
  }
};
struct GlobAcc {
  double* p;
  int nx, ny, nz;
  __device__ __forceinline__ static int wrap(int i, int n) {
    return i < 0 ? i + n : (i >= n ? i - n : i);
  }
  __device__ __forceinline__ void add(int i, int j, int k, double v) const {
    i = wrap(i, nx); j = wrap(j, ny); k = wrap(k, nz);
    atomicAdd(p + i + (i64)nx * (j + (i64)ny * k), v);
  }
};

// Esirkepov current of one particle into three accumulators, box in the
// accumulator's coordinates.  Same arithmetic as esirkepov_3d.F90 (prefix
// sums of W along x for Jx, y for Jy, z for Jz).
template <int ORDER, typename R, typename ACC, typename AV>
__device__ __forceinline__ void esirkepov_dep(const EsirAxis<ORDER, R>& X,
                                              const EsirAxis<ORDER, R>& Y,
                                              const EsirAxis<ORDER, R>& Z, R wqx, R wqy, R wqz,
                                              const ACC& jx, const ACC& jy, const ACC& jz) {
  constexpr int M = ORDER + 2;
  const R onethird = (R)(1.0 / 3.0);
#pragma unroll
  for (int k = 0; k < M; ++k) {
    if (k >= Z.n) continue;
    R dsz = Z.s1[k] - Z.s0[k];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      if (j >= Y.n) continue;
      R dsy = Y.s1[j] - Y.s0[j];
      R fyz = (Y.s0[j] + (R)0.5 * dsy) * Z.s0[k] + ((R)0.5 * Y.s0[j] + onethird * dsy) * dsz;
      R acc = (R)0;
#pragma unroll
      for (int i = 0; i < M - 1; ++i) {
        if (i >= X.n - 1) continue;
        acc = acc + wqx * (X.s1[i] - X.s0[i]) * fyz;
        jx.add(X.i0 + i, Y.i0 + j, Z.i0 + k, (AV)acc);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < M; ++k) {
    if (k >= Z.n) continue;
    R dsz = Z.s1[k] - Z.s0[k];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      if (i >= X.n) continue;
      R dsx = X.s1[i] - X.s0[i];
      R fzx = (Z.s0[k] + (R)0.5 * dsz) * X.s0[i] + ((R)0.5 * Z.s0[k] + onethird * dsz) * dsx;
      R acc = (R)0;
#pragma unroll
      for (int j = 0; j < M - 1; ++j) {
        if (j >= Y.n - 1) continue;
        acc = acc + wqy * (Y.s1[j] - Y.s0[j]) * fzx;
        jy.add(X.i0 + i, Y.i0 + j, Z.i0 + k, (AV)acc);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < M; ++j) {
    if (j >= Y.n) continue;
    R dsy = Y.s1[j] - Y.s0[j];
#pragma unroll
    for (int i = 0; i < M; ++i) {
      if (i >= X.n) continue;
      R dsx = X.s1[i] - X.s0[i];
      R fxy = (X.s0[i] + (R)0.5 * dsx) * Y.s0[j] + ((R)0.5 * X.s0[i] + onethird * dsx) * dsy;
      R acc = (R)0;
#pragma unroll
      for (int k = 0; k < M - 1; ++k) {
        if (k >= Z.n - 1) continue;
        acc = acc + wqz * (Z.s1[k] - Z.s0[k]) * fxy;
        jz.add(X.i0 + i, Y.i0 + j, Z.i0 + k, (AV)acc);
      }
    }
  }
}

template <typename R>
__device__ __forceinline__ void cell_step(R& o, int& c, R du) {
  // o + du, split into cell shift and offset in [0,1)
  R on = o + du;
  R fl = floor(on);
  int s = (int)fl;
  R of = on - fl;
  if (of >= (R)1) { of = of - (R)1; s += 1; }
  o = of;
  c += s;
}


// Shared-memory current accumulators (MODE):
//  0  FP32 atomics;
//  1  int32 fixed point, one word (scale 2^29 / node bound);
//  2  64-bit fixed point as two native int32 words: the value X (an integer,
//     |X| <= 2^42 per node by the scale) is split X = hi*2^12 + lo with
//     lo in [0, 2^12); both words are summed with int32 atomics and the sums
//     cannot overflow (|sum hi| <= 2^30, sum lo < 2^32 for < 2^20 terms);
//  3  FP64 atomics (FP64 engine).
// Fixed-point sums are order-independent, so a tile's current does not
// depend on the atomics' ordering.
template <int MODE> struct Acc;
template <> struct Acc<0> {
  typedef float T;
  static constexpr int NW = 1;
  static constexpr double SCALE_BITS = 0.0;
  __device__ __forceinline__ static void add(float* p, float v, int) { atomicAdd(p, v); }
  __device__ __forceinline__ static double get(const float* p, int r, int) { return p[r]; }
};
template <> struct Acc<1> {
  typedef int T;
  static constexpr int NW = 1;
  static constexpr double SCALE_BITS = 536870912.0;   // 2^29 (2^28 at order 1, below)
  // v rounded to the nearest integer by adding 1.5 * 2^23: for |v| <= 2^22
  // the sum lies in [2^23, 2^24], where the float spacing is 1, so its low
  // mantissa bits are round(v) + 2^22 (round half to even, as
  // __float2int_rn).  One FADD and one integer subtract replace a
  // conversion instruction, which issues at a fraction of the FMA rate.
  // The scale keeps every contribution within 2^22: it is at most
  // SCALE_BITS / (L+H+3)^3, i.e. 2^28 / 64 at order 1 and 2^29 / 216 above.
  __device__ __forceinline__ static void add(int* p, float v, int) {
    const float t = v + 12582912.0f;
    atomicAdd(p, __float_as_int(t) - 0x4B400000);
  }
  __device__ __forceinline__ static double get(const int* p, int r, int) { return (double)p[r]; }
};
template <> struct Acc<2> {
  typedef int T;
  static constexpr int NW = 2;
  static constexpr double SCALE_BITS = 4398046511104.0;  // 2^42
  __device__ __forceinline__ static void add(int* p, float v, int V3) {
    const long long X = __float2ll_rn(v);
    atomicAdd(p, (int)(X >> 12));
    atomicAdd(reinterpret_cast<unsigned*>(p + V3), (unsigned)(X & 0xFFF));
  }
  __device__ __forceinline__ static double get(const int* p, int r, int V3) {
    return (double)p[r] * 4096.0 + (double)reinterpret_cast<const unsigned*>(p)[r + V3];
  }
};
template <> struct Acc<3> {
  typedef double T;
  static constexpr int NW = 1;
  static constexpr double SCALE_BITS = 0.0;
  __device__ __forceinline__ static void add(double* p, double v, int) { atomicAdd(p, v); }
  __device__ __forceinline__ static double get(const double* p, int r, int) { return p[r]; }
};

// Esirkepov deposit in outer-product form: for Jx,
//   J(i,j,k) += cx * C_x(i) * F_yz(j,k),  C_x(i) = sum_{i'<=i} (s1 - s0)_x(i'),
//   F_yz = (s0y + ds_y/2) s0z + (s0y/2 + ds_y/3) ds_z,
// which is the reference's prefix sum of W_x (esirkepov_3d.F90:198-233) with
// the common factor taken out.  Box offsets are compile-time; the boxes'
// origins are runtime.  Window variant: shared memory, strides SY, SZ.
template <int ORDER, typename R, int MODE, int SY, int SZ, int V>
__device__ __forceinline__ void dep_window(typename Acc<MODE>::T* Js, const EsirAxis<ORDER, R>& X,
                                           const EsirAxis<ORDER, R>& Y,
                                           const EsirAxis<ORDER, R>& Z, R cx, R cy, R cz) {
  constexpr int M = ORDER + 2;
  const R third = (R)(1.0 / 3.0);
  typename Acc<MODE>::T* bx = Js + X.i0 + Y.i0 * SY + Z.i0 * SZ;
  typename Acc<MODE>::T* by = bx + V;
  typename Acc<MODE>::T* bz = bx + 2 * V;
#pragma unroll
  for (int k = 0; k < M; ++k) {
    if (k >= Z.n) continue;
    const R s0z = Z.s0[k], dsz = Z.s1[k] - s0z;
#pragma unroll
    for (int j = 0; j < M; ++j) {
      if (j >= Y.n) continue;
      const R s0y = Y.s0[j], dsy = Y.s1[j] - s0y;
      const R f = ((s0y + (R)0.5 * dsy) * s0z + ((R)0.5 * s0y + third * dsy) * dsz) * cx;
      R C = (R)0;
#pragma unroll
      for (int i = 0; i < M - 1; ++i) {
        if (i >= X.n - 1) continue;
        C += X.s1[i] - X.s0[i];
        Acc<MODE>::add(bx + i + j * SY + k * SZ, C * f, 3 * V);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < M; ++k) {
    if (k >= Z.n) continue;
    const R s0z = Z.s0[k], dsz = Z.s1[k] - s0z;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      if (i >= X.n) continue;
      const R s0x = X.s0[i], dsx = X.s1[i] - s0x;
      const R f = ((s0z + (R)0.5 * dsz) * s0x + ((R)0.5 * s0z + third * dsz) * dsx) * cy;
      R C = (R)0;
#pragma unroll
      for (int j = 0; j < M - 1; ++j) {
        if (j >= Y.n - 1) continue;
        C += Y.s1[j] - Y.s0[j];
        Acc<MODE>::add(by + i + j * SY + k * SZ, C * f, 3 * V);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < M; ++j) {
    if (j >= Y.n) continue;
    const R s0y = Y.s0[j], dsy = Y.s1[j] - s0y;
#pragma unroll
    for (int i = 0; i < M; ++i) {
      if (i >= X.n) continue;
      const R s0x = X.s0[i], dsx = X.s1[i] - s0x;
      const R f = ((s0x + (R)0.5 * dsx) * s0y + ((R)0.5 * s0x + third * dsx) * dsy) * cz;
      R C = (R)0;
#pragma unroll
      for (int k = 0; k < M - 1; ++k) {
        if (k >= Z.n - 1) continue;
        C += Z.s1[k] - Z.s0[k];
        Acc<MODE>::add(bz + i + j * SY + k * SZ, C * f, 3 * V);
      }
    }
  }
}

// Fast path of the window deposit: no node change along any axis (the common
// case), box of ORDER+1 nodes per axis starting at `base`; t0 = shape at the
// new position, t1 = shape at the old position on the same nodes.
template <int ORDER, typename R, int MODE, int SY, int SZ, int V>
__device__ __forceinline__ void dep_window_same(typename Acc<MODE>::T* base, const R* t0x,
                                                const R* t1x, const R* t0y, const R* t1y,
                                                const R* t0z, const R* t1z, R cx, R cy, R cz) {
  constexpr int N = ORDER + 1;
  const R third = (R)(1.0 / 3.0);
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const R s0z = t0z[k], dsz = t1z[k] - s0z;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const R s0y = t0y[j], dsy = t1y[j] - s0y;
      const R f = ((s0y + (R)0.5 * dsy) * s0z + ((R)0.5 * s0y + third * dsy) * dsz) * cx;
      R C = (R)0;
#pragma unroll
      for (int i = 0; i < N - 1; ++i) {
        C += t1x[i] - t0x[i];
        Acc<MODE>::add(base + i + j * SY + k * SZ, C * f, 3 * V);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const R s0z = t0z[k], dsz = t1z[k] - s0z;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const R s0x = t0x[i], dsx = t1x[i] - s0x;
      const R f = ((s0z + (R)0.5 * dsz) * s0x + ((R)0.5 * s0z + third * dsz) * dsx) * cy;
      R C = (R)0;
#pragma unroll
      for (int j = 0; j < N - 1; ++j) {
        C += t1y[j] - t0y[j];
        Acc<MODE>::add(base + V + i + j * SY + k * SZ, C * f, 3 * V);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const R s0y = t0y[j], dsy = t1y[j] - s0y;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const R s0x = t0x[i], dsx = t1x[i] - s0x;
      const R f = ((s0x + (R)0.5 * dsx) * s0y + ((R)0.5 * s0x + third * dsx) * dsy) * cz;
      R C = (R)0;
#pragma unroll
      for (int k = 0; k < N - 1; ++k) {
        C += t1z[k] - t0z[k];
        Acc<MODE>::add(base + 2 * V + i + j * SY + k * SZ, C * f, 3 * V);
      }
    }
  }
}

// Global variant (particles outside their tile window): FP64 atomics on the
// periodic J grid, in the reference's W-prefix form (unscaled coefficients).
template <int ORDER, typename R>
__device__ __noinline__ void dep_global(const Job& J, const EsirAxis<ORDER, R>& X,
                                        const EsirAxis<ORDER, R>& Y,
                                        const EsirAxis<ORDER, R>& Z, R cx, R cy, R cz) {
  GlobAcc G[3];
  G[0].p = J.jx; G[1].p = J.jy; G[2].p = J.jz;
  for (int c = 0; c < 3; ++c) { G[c].nx = J.nx; G[c].ny = J.ny; G[c].nz = J.nz; }
  esirkepov_dep<ORDER, R, GlobAcc, double>(X, Y, Z, cx, cy, cz, G[0], G[1], G[2]);
}

template <int ORDER, typename R>
__device__ __noinline__ void gather_global(const Job& J, int ci, int cj, int ck, R ox, R oy,
                                           R oz, R* eb) {
  const int G = J.g, pitch = J.pitch_x, NYg = J.pitch_y;
  FieldView<R> F[6];
  const void* src[6] = {J.ex, J.ey, J.ez, J.bx, J.by, J.bz};
  for (int c = 0; c < 6; ++c) {
    F[c].p = (const R*)src[c] + (G + (i64)pitch * (G + (i64)NYg * G));
    F[c].sy = pitch; F[c].sz = pitch * NYg;
  }
  gather6<ORDER, R>(F, ci, cj, ck, ox, oy, oz, eb);
}

// Gather from the shared window with compile-time strides: each component's
// support starts at `base`, points at base + t + b*SY + c*SZ.
template <int NA, int NB, int NC, int SY, int SZ, typename R>
__device__ __forceinline__ R gwin(const R* base, const R* sa, const R* sb, const R* sc) {
  R out = (R)0;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    R a = (R)0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      R r = (R)0;
#pragma unroll
      for (int t = 0; t < NA; ++t) r = r + sa[t] * base[t + b * SY + c * SZ];
      a = a + r * sb[b];
    }
    out = out + a * sc[c];
  }
  return out;
}

// Fixed-point resolution of a mode: the largest node sum, as an integer.
template <int MODE, int ORDER> __host__ __device__ constexpr double scale_bits() {
  return (MODE == 1 && ORDER == 1) ? 268435456.0 : Acc<MODE>::SCALE_BITS;   // 2^28
}

// ---------------------------------------------------------------------------
// Packed FP32 pairs (sm_100 fma/mul .f32x2): one instruction performs two
// independent single-precision operations, each rounded as its scalar form.
// ---------------------------------------------------------------------------
typedef unsigned long long f2_t;
__device__ __forceinline__ f2_t f2_pack(float lo, float hi) {
  f2_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float f2_sum(f2_t v) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
  return lo + hi;
}
__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c) {
  f2_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f2_t f2_mul(f2_t a, f2_t b) {
  f2_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// FP32 window gather with the z-planes taken in pairs: each packed FMA
// advances two planes' sums, so the point sums of a component take
// NA*NB*ceil(NC/2) instructions instead of NA*NB*NC.  An odd last plane is
// summed in scalar form.  The per-plane sums are those of gwin; only the
// final sum over the planes is ordered differently.
template <int NA, int NB, int NC, int SY, int SZ>
__device__ __forceinline__ float gwin2(const float* base, const f2_t* sa2, const f2_t* sb2,
                                       const float* sc) {
  f2_t out2 = f2_pack(0.f, 0.f);
#pragma unroll
  for (int c = 0; c + 1 < NC; c += 2) {
    f2_t a2;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      f2_t r2 = f2_mul(f2_pack(base[b * SY + c * SZ], base[b * SY + (c + 1) * SZ]), sa2[0]);
#pragma unroll
      for (int t = 1; t < NA; ++t)
        r2 = f2_fma(f2_pack(base[t + b * SY + c * SZ], base[t + b * SY + (c + 1) * SZ]), sa2[t], r2);
      a2 = b == 0 ? f2_mul(r2, sb2[0]) : f2_fma(r2, sb2[b], a2);
    }
    out2 = f2_fma(a2, f2_pack(sc[c], sc[c + 1]), out2);
  }
  float out = f2_sum(out2);
  if (NC & 1) {
    constexpr int c = NC - 1;
    float a = 0.f;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      float r = 0.f;
#pragma unroll
      for (int t = 0; t < NA; ++t) {
        float sat, dummy;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(sat), "=f"(dummy) : "l"(sa2[t]));
        r = r + sat * base[t + b * SY + c * SZ];
      }
      float sbb, dummy2;
      asm("mov.b64 {%0, %1}, %2;" : "=f"(sbb), "=f"(dummy2) : "l"(sb2[b]));
      a = a + r * sbb;
    }
    out = out + a * sc[c];
  }
  return out;
}

template <int N>
__device__ __forceinline__ void f2_splat(const float* s, f2_t* s2) {
#pragma unroll
  for (int i = 0; i < N; ++i) s2[i] = f2_pack(s[i], s[i]);
}

constexpr int MAX_THREADS = 256;        // FP32 engine: two CTAs per SM
constexpr int MAX_THREADS_FP64 = 512;   // FP64 engine: one CTA per SM
constexpr int MAX_WARPS = MAX_THREADS_FP64 / 32;

// Window particles whose Esirkepov node changes along some axis are queued
// and deposited after the tile's main loop by full warps, so the common
// same-node path never diverges into the general one.  The queue lives in
// the sort's scratch buffers, free between sorts: the tile's own range of
// rank_b lists the queued particles, and each queued particle's slot of
// ox_b/oy_b/oz_b and cell_b holds its old offsets and packed box - so the
// queue holds every particle of the tile and cannot overflow.

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

// ---------------------------------------------------------------------------
// The fused particle kernel.  Persistent CTAs pull (job, tile) work items;
// tile edge T (cells), window margin D: compile-time, so every shared-memory
// address of the gather and of the deposition is a register plus an
// immediate.  Windows of partial tiles extend into the padded guard region of
// the field arrays (never written, zero) which no particle reaches.
// ---------------------------------------------------------------------------
// FP32 windows fit two CTAs of 256 threads per SM (128 registers per
// thread); the FP64 engine's windows take one CTA per SM, of up to 512
// threads (128 registers): its FP64 shared atomics want the warps (256 /
// 384 / 512 / 640 threads measured 76.6 / 63.5 / 58.0 / 58.8 ms at 256^3).
template <typename R, int ORDER, int T, int D, int MODE>
__global__ void __launch_bounds__(sizeof(R) == 8 ? MAX_THREADS_FP64 : MAX_THREADS,
                                  sizeof(R) == 8 ? 1 : 2)
    k_tile_step(const Job* __restrict__ jobs, const int2* __restrict__ work, int nwork,
                const int* __restrict__ nwork_dev, int* ctr) {
  constexpr int L = Reach<ORDER>::L, H = Reach<ORDER>::H;
  constexpr int W = T + 2 * D + L + H, SY = win_sy(T, W), SZ = win_sz(T, W), V = SZ * W;
  typedef typename Acc<MODE>::T A;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* Fs = reinterpret_cast<R*>(smem_raw);
  A* Js = reinterpret_cast<A*>(smem_raw + (size_t)6 * V * sizeof(R));
  constexpr bool FIXED = MODE == 1 || MODE == 2;
  // occupancy of the window cells after this step, for the next step's scale
  constexpr int HB = T + 2 * D;
  int* nh = reinterpret_cast<int*>(Js + 3 * V * Acc<MODE>::NW);
  __shared__ int s_have;
  __shared__ Job sj;
  __shared__ int s_item;
  __shared__ int s_qn;
  // bank-conflict-free pass selection (FP32 windows; see the particle loop)
  constexpr bool SELECT = sizeof(R) == 4;
  __shared__ int s_dn;                             // deferred particles of the tile
  __shared__ int s_dcnt[32];                       // ... per bank class
  __shared__ float s_max[5][MAX_WARPS];
  __shared__ double s_red[MAX_WARPS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;

  if (nwork_dev) nwork = min(nwork, *nwork_dev);
  // the window's pitch padding is never staged: zero it once, so that whole
  // components can be scanned without decoding window coordinates
  for (int r = threadIdx.x; r < 6 * V; r += blockDim.x) {
    const int q = r % V, c = q / SZ, b = (q - c * SZ) / SY, a = q - c * SZ - b * SY;
    if (a >= W || b >= W) Fs[r] = (R)0;
  }
  for (;;) {
    if (threadIdx.x == 0) {
      s_item = atomicAdd(ctr, 1);
      s_qn = 0;
      s_dn = 0;
    }
    __syncthreads();
    const int item = s_item;
    if (item >= nwork) break;
    const int2 wk = work[item];
    {
      const int nw = (int)(sizeof(Job) / sizeof(int));
      const int* src = reinterpret_cast<const int*>(jobs + wk.x);
      int* dst = reinterpret_cast<int*>(&sj);
      for (int t = threadIdx.x; t < nw; t += blockDim.x) dst[t] = src[t];
    }
    __syncthreads();
    const int nx = sj.nx, ny = sj.ny, nz = sj.nz, G = sj.g;
    const int tile = wk.y;
    const int ti = tile % sj.ntx, tj = (tile / sj.ntx) % sj.nty, tk = tile / (sj.ntx * sj.nty);
    const int c0x = ti * T, c0y = tj * T, c0z = tk * T;
    const int tex = min(T, nx - c0x), tey = min(T, ny - c0y), tez = min(T, nz - c0z);
    const int wox = c0x - D - L, woy = c0y - D - L, woz = c0z - D - L;
    const int pbeg = sj.tile_off[tile], pend = sj.tile_off[tile + 1];
    // ---- stage the E/B window: asynchronous copies (cp.async), in flight
    // while the accumulator is cleared and the tile's bounds are gathered ----
    const int pitch = sj.pitch_x, NYg = sj.pitch_y;
    {
      const i64 base0 = (i64)(wox + G) + (i64)pitch * ((woy + G) + (i64)NYg * (woz + G));
#pragma unroll 1
      for (int comp = 0; comp < 6; ++comp) {
        const R* src = (const R*)(comp == 0 ? sj.ex : comp == 1 ? sj.ey : comp == 2 ? sj.ez
                                 : comp == 3 ? sj.bx : comp == 4 ? sj.by : sj.bz) + base0;
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(Fs + comp * V);
        for (int r = threadIdx.x; r < W * W * W; r += blockDim.x) {
          const int a = r % W, b = (r / W) % W, c = r / (W * W);
          const R* g = src + a + (i64)pitch * (b + (i64)NYg * c);
          const uint32_t d = dst + (uint32_t)((a + b * SY + c * SZ) * sizeof(R));
          asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(g),
                       "n"((int)sizeof(R)));
        }
      }
      asm volatile("cp.async.commit_group;\n" ::);
    }
    {
      // 16-byte stores where the accumulator's size and offset allow
      constexpr size_t JB = (size_t)3 * V * Acc<MODE>::NW * sizeof(A);
      constexpr bool VEC = JB % 16 == 0 && ((size_t)6 * V * sizeof(R)) % 16 == 0;
      if (VEC) {
        uint4* j4 = reinterpret_cast<uint4*>(Js);
        for (int e = threadIdx.x; e < (int)(JB / 16); e += blockDim.x) j4[e] = make_uint4(0, 0, 0, 0);
      } else {
        for (int e = threadIdx.x; e < 3 * V * Acc<MODE>::NW; e += blockDim.x) Js[e] = (A)0;
      }
    }
    if (FIXED)
      for (int e = threadIdx.x; e < HB * HB * HB; e += blockDim.x) nh[e] = 0;
    float* stats = FIXED && sj.tile_stats ? sj.tile_stats + 4 * (size_t)tile : nullptr;
    if (threadIdx.x == 0) s_have = stats && stats[3] != 0.f;
    // ---- fixed-point scale of the current window (FP32 engine) -------------
    // Bound of one particle's contribution to one node of J_c:
    //   |q| w_max / (dt dV / d_c) * (max displacement along c in cells),
    // with the displacement bounded from max |u| of the tile's particles
    // before the push and the largest change the push can make to |u| in
    // the window's fields (below).
    // A node of the window receives deposits only from particles whose old
    // cell lies within L+H+3 cells of it along every axis, so the node sum
    // is bounded by (max particles per window cell) * (L+H+3)^3 contributions.
    // The bounds are carried from the previous step of this tile (written at
    // its end for the same particles in their new cells), or, after a sort,
    // taken by a pre-pass over the tile's particles.
    float umax2 = 0.f, wmax = 0.f, cmax = 0.f;
    __syncthreads();
    const bool have = FIXED && s_have;
    if (have) {
      umax2 = stats[0]; wmax = stats[1]; cmax = stats[2];
    } else if (FIXED) {
      int* hist = reinterpret_cast<int*>(Js) + 2 * V;   // zero; re-zeroed below
      const R* uxp = (const R*)sj.ux; const R* uyp = (const R*)sj.uy;
      const R* uzp = (const R*)sj.uz; const R* wp = (const R*)sj.w;
      for (int ip = pbeg + threadIdx.x; ip < pend; ip += blockDim.x) {
        float a = (float)uxp[ip], b = (float)uyp[ip], c = (float)uzp[ip];
        umax2 = fmaxf(umax2, a * a + b * b + c * c);
        wmax = fmaxf(wmax, fabsf((float)wp[ip]));
        int ci, cj, ck;
        unpack_cell(sj.cell[ip], ci, cj, ck);
        int vx = ci - c0x, vy = cj - c0y, vz = ck - c0z;
        if (vx > tex - 1 + D) vx -= nx; else if (vx < -D) vx += nx;
        if (vy > tey - 1 + D) vy -= ny; else if (vy < -D) vy += ny;
        if (vz > tez - 1 + D) vz -= nz; else if (vz < -D) vz += nz;
        if (vx >= -D && vx <= tex - 1 + D && vy >= -D && vy <= tey - 1 + D && vz >= -D &&
            vz <= tez - 1 + D)
          atomicAdd(hist + (vx + D + L) + (vy + D + L) * SY + (vz + D + L) * SZ, 1);
      }
      __syncthreads();
      for (int r = threadIdx.x; r < V; r += blockDim.x) {
        cmax = fmaxf(cmax, (float)hist[r]);
        hist[r] = 0;
      }
    }
    // ---- window staged: |E|, |B| maxima ---------------------------------------
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    float emax = 0.f, bmax = 0.f;
    if (sizeof(R) == 4 && (3 * V) % 4 == 0) {     // 16-byte loads
      const float4* e4 = reinterpret_cast<const float4*>(Fs);
      const float4* b4 = e4 + (3 * V) / 4;
      for (int r = threadIdx.x; r < (3 * V) / 4; r += blockDim.x) {
        const float4 e = e4[r], b = b4[r];
        emax = fmaxf(emax, fmaxf(fmaxf(fabsf(e.x), fabsf(e.y)), fmaxf(fabsf(e.z), fabsf(e.w))));
        bmax = fmaxf(bmax, fmaxf(fmaxf(fabsf(b.x), fabsf(b.y)), fmaxf(fabsf(b.z), fabsf(b.w))));
      }
    } else {
      for (int r = threadIdx.x; r < 3 * V; r += blockDim.x) {
        emax = fmaxf(emax, fabsf((float)Fs[r]));
        bmax = fmaxf(bmax, fabsf((float)Fs[r + 3 * V]));
      }
    }
    emax = warp_max(emax); bmax = warp_max(bmax); umax2 = warp_max(umax2); wmax = warp_max(wmax);
    cmax = warp_max(cmax);
    if (lane == 0) {
      s_max[0][wid] = emax; s_max[1][wid] = bmax; s_max[2][wid] = umax2; s_max[3][wid] = wmax;
      s_max[4][wid] = cmax;
    }
    __syncthreads();
    double scale[3];
    scale[0] = scale[1] = scale[2] = 1.0;
    if (FIXED) {
      float E = 0.f, B = 0.f, U2 = 0.f, Wm = 0.f, Cm = 0.f;
      for (int w = 0; w < nwarps; ++w) {
        E = fmaxf(E, s_max[0][w]); B = fmaxf(B, s_max[1][w]);
        U2 = fmaxf(U2, s_max[2][w]); Wm = fmaxf(Wm, s_max[3][w]); Cm = fmaxf(Cm, s_max[4][w]);
      }
      const double c = sj.clight;
      // |u| after the push, from |u| before it (U2) and the window maxima of
      // |E| and |B| (componentwise maxima, times sqrt 3).  With qdm = |q| dt / m
      // and tau = qdm |B| / 2 (the rotation parameter of both pushers): Boris
      // changes |u| only by its two half E kicks, |u'| <= |u| + qdm |E|; Vay
      // gives |u + qdm E + (u x tau) / gamma| <= |u| (1 + tau) + qdm |E| before
      // its rotation and scales that by at most (1 + t + t^2) / (1 + t^2) <=
      // 1 + tau.  So |u'| <= (|u| (1 + tau) + qdm |E|) (1 + tau) bounds both; the
      // last factor covers the FP32 rounding of the pushers.
      const double qdm = fabs(sj.q) / sj.m * sj.dt;
      const double tau = 0.5 * qdm * 1.7320508075688772 * (double)B;
      const double ub = (sqrt((double)U2) * (1.0 + tau) + qdm * 1.7320508075688772 * (double)E) *
                        (1.0 + tau) * 1.0001;
      const double vb = ub / sqrt(1.0 + ub * ub / (c * c));
      const double dV = sj.dx * sj.dy * sj.dz;
      constexpr int reach = L + H + 3;
      const double np_ = fmax((double)Cm * (reach * reach * reach), 1.0);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const double dq = q == 0 ? sj.dx : (q == 1 ? sj.dy : sj.dz);
        const double disp = fmin(vb * sj.dt / dq, 1.0);
        const double bound = fabs(sj.q) * (double)Wm * dq / (sj.dt * dV) * disp;
        const double s = scale_bits<MODE, ORDER>() / fmax(np_ * bound, 1e-300);
        scale[q] = fmin(s, 1e30);
      }
    }
    // ---- particles -----------------------------------------------------------
    const R dtdx = (R)(sj.dt / sj.dx), dtdy = (R)(sj.dt / sj.dy), dtdz = (R)(sj.dt / sj.dz);
    const R clghtisq = (R)(1.0 / (sj.clight * sj.clight));
    const R cst_b = (R)(sj.q * sj.dt * 0.5 / sj.m), cst_v = (R)(sj.q * sj.dt / sj.m);
    const R invc = (R)(1.0 / sj.clight);
    const R qdx = (R)(sj.q / (sj.dt * sj.dy * sj.dz)), qdy = (R)(sj.q / (sj.dt * sj.dx * sj.dz)),
            qdz = (R)(sj.q / (sj.dt * sj.dx * sj.dy));
    const R scx = (R)scale[0], scy = (R)scale[1], scz = (R)scale[2];
    const bool vay = sj.pusher == 1;
    uint32_t* cellp = sj.cell;
    R *oxp = (R*)sj.ox, *oyp = (R*)sj.oy, *ozp = (R*)sj.oz;
    R *uxp = (R*)sj.ux, *uyp = (R*)sj.uy, *uzp = (R*)sj.uz;
    const R* wp = (const R*)sj.w;
    int* q_list = sj.rank_b;
    uint32_t* q_pk = sj.cell_b;
    R *q_ox = (R*)sj.ox_b, *q_oy = (R*)sj.oy_b, *q_oz = (R*)sj.oz_b;
    double ke = 0.0;
    float nu2 = 0.f, nwm = 0.f;          // the next step's bounds (fixed point)
    int nslow = 0, bad = 0;
    __syncthreads();

    // Two passes over the tile.  Pass 0 takes the particles in storage
    // order, 32 consecutive ones per warp; a window particle whose bank class
    // (the bank of its stencil origin in the window, so of every one of its
    // gather loads and fast-path atomics) a lower lane of the warp already
    // holds is deferred, so every warp instruction of the pass reads or
    // updates 32 distinct banks whatever the particles' drift since the last
    // sort.  Pass 1 takes the deferred particles bucketed by class, in
    // (rank, class) order, so its warps too hold distinct classes except at
    // the tail.  FP32 windows only (one 4-byte bank per element); the FP64
    // engine makes one pass.  The deferred list, its classes and its
    // bucketed order live in the tile's range of sort scratch that is free
    // between sorts: perm, and ux_b / uy_b / uz_b taken as integers.
    int* d_list = sj.perm;
    int* d_ord = reinterpret_cast<int*>(sj.ux_b);
    int* d_rank = reinterpret_cast<int*>(sj.uy_b);
    int* d_key = reinterpret_cast<int*>(sj.uz_b);
#pragma unroll 1
    for (int phase = 0; phase < (SELECT ? 2 : 1); ++phase) {
    const int cnt = phase == 0 ? pend - pbeg : s_dn;
    for (int s0 = threadIdx.x & ~31; s0 < cnt; s0 += blockDim.x) {
      const int sl = s0 + lane;
      const bool valid = sl < cnt;
      // lanes past the end read a valid particle and do nothing with it
      const int slc = valid ? sl : 0;
      const int ip = phase == 0 ? pbeg + slc : d_list[pbeg + d_ord[pbeg + slc]];
      int ci, cj, ck;
      unpack_cell(cellp[ip], ci, cj, ck);
      const R ox = oxp[ip], oy = oyp[ip], oz = ozp[ip];
      R ux = uxp[ip], uy = uyp[ip], uz = uzp[ip];
      const R wgt = wp[ip];
      int vx = ci - c0x, vy = cj - c0y, vz = ck - c0z;
      if (vx > tex - 1 + D) vx -= nx; else if (vx < -D) vx += nx;
      if (vy > tey - 1 + D) vy -= ny; else if (vy < -D) vy += ny;
      if (vz > tez - 1 + D) vz -= nz; else if (vz < -D) vz += nz;
      const bool in_old = vx >= -D && vx <= tex - 1 + D && vy >= -D && vy <= tey - 1 + D &&
                          vz >= -D && vz <= tez - 1 + D;
      if (SELECT && phase == 0 && sj.select_lanes) {
        const bool part = valid && in_old;
        const int hx = ORDER == 2 && ox >= (R)0.5, hy = ORDER == 2 && oy >= (R)0.5,
                  hz = ORDER == 2 && oz >= (R)0.5;
        const int key = (vx + hx + (vy + hy) * SY + (vz + hz) * SZ + (D + L) * (1 + SY + SZ)) & 31;
        // lanes holding the same class: five ballots over the class bits
        unsigned peers = __ballot_sync(0xffffffffu, part);
#pragma unroll
        for (int b = 0; b < 5; ++b) {
          const unsigned m = __ballot_sync(0xffffffffu, part && ((key >> b) & 1));
          peers &= ((key >> b) & 1) ? m : ~m;
        }
        if (part && (peers & ((1u << lane) - 1u))) {
          const int q = atomicAdd(&s_dn, 1);
          d_list[pbeg + q] = ip;
          d_key[pbeg + q] = key;
          continue;
        }
      }
      if (!valid) continue;
      // ---- gather ----------------------------------------------------------
      R eb[6];
      if (in_old) {
        const int wx = vx + D + L, wy = vy + D + L, wz = vz + D + L;
        NodeCO<ORDER, R> nxs, nys, nzs;
        StagCO<ORDER, R> sxs, sys, szs;
        nxs.set(ox); nys.set(oy); nzs.set(oz);
        sxs.set(ox); sys.set(oy); szs.set(oz);
        constexpr int N = ORDER + 1, S = ORDER;
        const R* F0 = Fs + wx + wy * SY + wz * SZ;
        if constexpr (sizeof(R) == 4 && ORDER > 1) {
          // x and y shapes splatted once into packed pairs for the z-plane pairs
          f2_t nx2[N], sx2[S], ny2[N], sy2[S];
          f2_splat<N>((const float*)nxs.s, nx2); f2_splat<S>((const float*)sxs.s, sx2);
          f2_splat<N>((const float*)nys.s, ny2); f2_splat<S>((const float*)sys.s, sy2);
          const float* Ff = (const float*)F0;
          eb[0] = gwin2<S, N, N, SY, SZ>(Ff + sxs.r0 + nys.r0 * SY + nzs.r0 * SZ, sx2, ny2, (const float*)nzs.s);
          eb[1] = gwin2<N, S, N, SY, SZ>(Ff + V + nxs.r0 + sys.r0 * SY + nzs.r0 * SZ, nx2, sy2, (const float*)nzs.s);
          eb[2] = gwin2<N, N, S, SY, SZ>(Ff + 2 * V + nxs.r0 + nys.r0 * SY + szs.r0 * SZ, nx2, ny2, (const float*)szs.s);
          eb[3] = gwin2<N, S, S, SY, SZ>(Ff + 3 * V + nxs.r0 + sys.r0 * SY + szs.r0 * SZ, nx2, sy2, (const float*)szs.s);
          eb[4] = gwin2<S, N, S, SY, SZ>(Ff + 4 * V + sxs.r0 + nys.r0 * SY + szs.r0 * SZ, sx2, ny2, (const float*)szs.s);
          eb[5] = gwin2<S, S, N, SY, SZ>(Ff + 5 * V + sxs.r0 + sys.r0 * SY + nzs.r0 * SZ, sx2, sy2, (const float*)nzs.s);
        } else {
          eb[0] = gwin<S, N, N, SY, SZ>(F0 + sxs.r0 + nys.r0 * SY + nzs.r0 * SZ, sxs.s, nys.s, nzs.s);
          eb[1] = gwin<N, S, N, SY, SZ>(F0 + V + nxs.r0 + sys.r0 * SY + nzs.r0 * SZ, nxs.s, sys.s, nzs.s);
          eb[2] = gwin<N, N, S, SY, SZ>(F0 + 2 * V + nxs.r0 + nys.r0 * SY + szs.r0 * SZ, nxs.s, nys.s, szs.s);
          eb[3] = gwin<N, S, S, SY, SZ>(F0 + 3 * V + nxs.r0 + sys.r0 * SY + szs.r0 * SZ, nxs.s, sys.s, szs.s);
          eb[4] = gwin<S, N, S, SY, SZ>(F0 + 4 * V + sxs.r0 + nys.r0 * SY + szs.r0 * SZ, sxs.s, nys.s, szs.s);
          eb[5] = gwin<S, S, N, SY, SZ>(F0 + 5 * V + sxs.r0 + sys.r0 * SY + nzs.r0 * SZ, sxs.s, sys.s, nzs.s);
        }
      } else {
        gather_global<ORDER, R>(sj, ci, cj, ck, ox, oy, oz, eb);
      }
      // ---- push ------------------------------------------------------------
      R gi;
      if (vay) {
        gi = inv_sqrt<R>((R)1 + (ux * ux + uy * uy + uz * uz) * clghtisq);
        vay_push(ux, uy, uz, gi, eb[0], eb[1], eb[2], eb[3], eb[4], eb[5], cst_v, invc, clghtisq);
      } else {
        boris_push(ux, uy, uz, gi, eb[0], eb[1], eb[2], eb[3], eb[4], eb[5], cst_b, clghtisq);
        set_gamma(ux, uy, uz, gi, clghtisq);
      }
      // ---- position: exact old (c, o) -> new (c + s, o') ----------------------
      R nox = ox, noy = oy, noz = oz;
      int sx = 0, sy = 0, sz = 0;
      cell_step(nox, sx, ux * gi * dtdx);
      cell_step(noy, sy, uy * gi * dtdy);
      cell_step(noz, sz, uz * gi * dtdz);
      const bool in_new = in_old && vx + sx >= -D && vx + sx <= tex - 1 + D &&
                          vy + sy >= -D && vy + sy <= tey - 1 + D && vz + sz >= -D &&
                          vz + sz <= tez - 1 + D;
      // ---- deposition --------------------------------------------------------
      {
        int r0x, r1x, r0y, r1y, r0z, r1z;
        R x0, x1, y0, y1, z0, z1;
        esir_node<ORDER, R>(nox, r0x, x0); esir_node<ORDER, R>(ox, r1x, x1);
        esir_node<ORDER, R>(noy, r0y, y0); esir_node<ORDER, R>(oy, r1y, y1);
        esir_node<ORDER, R>(noz, r0z, z0); esir_node<ORDER, R>(oz, r1z, z1);
        // node indices relative to the old cell: new = shift + r0, old = r1
        const bool same = (sx + r0x == r1x) && (sy + r0y == r1y) && (sz + r0z == r1z);
        const R wq = wgt;
        if (in_new && same) {
          constexpr int a = ORDER / 2;
          R t0x[ORDER + 1], t1x[ORDER + 1], t0y[ORDER + 1], t1y[ORDER + 1], t0z[ORDER + 1],
              t1z[ORDER + 1];
          EsirAxis<ORDER, R>::shape(x0, t0x); EsirAxis<ORDER, R>::shape(x1, t1x);
          EsirAxis<ORDER, R>::shape(y0, t0y); EsirAxis<ORDER, R>::shape(y1, t1y);
          EsirAxis<ORDER, R>::shape(z0, t0z); EsirAxis<ORDER, R>::shape(z1, t1z);
          A* base = Js + (vx + D + L + r1x - a) + (vy + D + L + r1y - a) * SY +
                    (vz + D + L + r1z - a) * SZ;
          dep_window_same<ORDER, R, MODE, SY, SZ, V>(base, t0x, t1x, t0y, t1y, t0z, t1z,
                                                     wq * qdx * scx, wq * qdy * scy,
                                                     wq * qdz * scz);
        } else {
          const int bx = in_new ? vx + D + L : ci;
          const int by = in_new ? vy + D + L : cj;
          const int bz = in_new ? vz + D + L : ck;
          EsirAxis<ORDER, R> EX, EY, EZ;
          bool ok = EX.set(bx + sx + r0x, x0, bx + r1x, x1);
          ok = EY.set(by + sy + r0y, y0, by + r1y, y1) && ok;
          ok = EZ.set(bz + sz + r0z, z0, bz + r1z, z1) && ok;
          if (!ok) bad = 1;
          if (in_new) {
            const int q = atomicAdd(&s_qn, 1);
            q_list[pbeg + q] = ip;
            q_pk[ip] = (unsigned)(vx + D + L) | ((unsigned)(vy + D + L) << 8) |
                       ((unsigned)(vz + D + L) << 16) | ((unsigned)(sx + 1) << 24) |
                       ((unsigned)(sy + 1) << 26) | ((unsigned)(sz + 1) << 28);
            q_ox[ip] = ox; q_oy[ip] = oy; q_oz[ip] = oz;
          } else {
            ++nslow;
            dep_global<ORDER, R>(sj, EX, EY, EZ, wq * qdx, wq * qdy, wq * qdz);
          }
        }
      }
      // ---- store -------------------------------------------------------------
      int nci = ci + sx, ncj = cj + sy, nck = ck + sz;
      nci = nci < 0 ? nci + nx : (nci >= nx ? nci - nx : nci);
      ncj = ncj < 0 ? ncj + ny : (ncj >= ny ? ncj - ny : ncj);
      nck = nck < 0 ? nck + nz : (nck >= nz ? nck - nz : nck);
      cellp[ip] = pack_cell(nci, ncj, nck);
      oxp[ip] = nox; oyp[ip] = noy; ozp[ip] = noz;
      uxp[ip] = ux; uyp[ip] = uy; uzp[ip] = uz;
      if (FIXED && stats) {
        // what the next step's pre-pass would find for this particle
        int hx = nci - c0x, hy = ncj - c0y, hz = nck - c0z;
        if (hx > tex - 1 + D) hx -= nx; else if (hx < -D) hx += nx;
        if (hy > tey - 1 + D) hy -= ny; else if (hy < -D) hy += ny;
        if (hz > tez - 1 + D) hz -= nz; else if (hz < -D) hz += nz;
        if (hx >= -D && hx <= tex - 1 + D && hy >= -D && hy <= tey - 1 + D && hz >= -D &&
            hz <= tez - 1 + D)
          atomicAdd(nh + (hx + D) + (hy + D) * HB + (hz + D) * (HB * HB), 1);
        const float a = (float)ux, b = (float)uy, c = (float)uz;
        nu2 = fmaxf(nu2, a * a + b * b + c * c);
        nwm = fmaxf(nwm, fabsf((float)wgt));
      }
      // kinetic energy (gamma - 1) w of the particle in the engine's precision,
      // summed over the tile in FP64
      {
        const R u2 = (ux * ux + uy * uy + uz * uz) * clghtisq;
        ke += (double)(quot<R>(u2, (R)1 + sqrt(u2 + (R)1)) * wgt);
      }
    }
    __syncthreads();
    if (SELECT && phase == 0 && s_dn > 0) {
      // bucket the deferred particles by class: the entry of rank r in class
      // k goes to sum_c min(n_c, r) + #{c < k : n_c > r}
      const int nd = s_dn;
      if (threadIdx.x < 32) s_dcnt[threadIdx.x] = 0;
      __syncthreads();
      for (int q = threadIdx.x; q < nd; q += blockDim.x)
        d_rank[pbeg + q] = atomicAdd(&s_dcnt[d_key[pbeg + q]], 1);
      __syncthreads();
      for (int q = threadIdx.x; q < nd; q += blockDim.x) {
        const int k = d_key[pbeg + q], r = d_rank[pbeg + q];
        int P = 0;
#pragma unroll 8
        for (int c = 0; c < 32; ++c) {
          const int n = s_dcnt[c];
          P += min(n, r) + (c < k && n > r ? 1 : 0);
        }
        d_ord[pbeg + P] = q;
      }
      __syncthreads();
    }
    }   // phase
    // ---- deferred window particles with a node change ------------------------
    {
      const int nq = s_qn;
      for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        const int ip = q_list[pbeg + q];
        const unsigned pk = q_pk[ip];
        const int bx = pk & 255u, by = (pk >> 8) & 255u, bz = (pk >> 16) & 255u;
        const int sx = (int)((pk >> 24) & 3u) - 1, sy = (int)((pk >> 26) & 3u) - 1,
                  sz = (int)((pk >> 28) & 3u) - 1;
        const R ox = q_ox[ip], oy = q_oy[ip], oz = q_oz[ip];
        const R nox = oxp[ip], noy = oyp[ip], noz = ozp[ip], wq = wp[ip];
        int r0, r1;
        R a0, a1;
        EsirAxis<ORDER, R> EX, EY, EZ;
        esir_node<ORDER, R>(nox, r0, a0); esir_node<ORDER, R>(ox, r1, a1);
        bool ok = EX.set(bx + sx + r0, a0, bx + r1, a1);
        esir_node<ORDER, R>(noy, r0, a0); esir_node<ORDER, R>(oy, r1, a1);
        ok = EY.set(by + sy + r0, a0, by + r1, a1) && ok;
        esir_node<ORDER, R>(noz, r0, a0); esir_node<ORDER, R>(oz, r1, a1);
        ok = EZ.set(bz + sz + r0, a0, bz + r1, a1) && ok;
        if (!ok) bad = 1;
        dep_window<ORDER, R, MODE, SY, SZ, V>(Js, EX, EY, EZ, wq * qdx * scx, wq * qdy * scy,
                                              wq * qdz * scz);
      }
    }
    __syncthreads();
    // ---- flush the J window: FP64 atomics into the periodic grid -------------
    {
#pragma unroll 1
      for (int comp = 0; comp < 3; ++comp) {
        double* dst = comp == 0 ? sj.jx : comp == 1 ? sj.jy : sj.jz;
        const double inv = 1.0 / (comp == 0 ? scale[0] : comp == 1 ? scale[1] : scale[2]);
        const A* src = Js + comp * V;
        for (int r = threadIdx.x; r < V; r += blockDim.x) {
          const double v = Acc<MODE>::get(src, r, 3 * V);
          if (v == 0.0) continue;               // includes the pitch padding
          const int c = r / SZ, b = (r - c * SZ) / SY, a = r - c * SZ - b * SY;
          const int gi = GlobAcc::wrap(wox + a, nx), gj = GlobAcc::wrap(woy + b, ny),
                    gk = GlobAcc::wrap(woz + c, nz);
          atomicAdd(dst + gi + (i64)nx * (gj + (i64)ny * gk), v * inv);
        }
      }
    }
    // ---- kinetic energy of the tile ------------------------------------------
    {
      double v = ke;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) s_red[wid] = v;
      if (nslow) atomicAdd(&sj.counters[0], nslow);
      if (bad) atomicExch(&sj.counters[1], 1);
      if (SELECT && threadIdx.x == 0 && s_dn) atomicAdd(&sj.counters[2], s_dn);
      if (FIXED && stats) {
        float c = 0.f;
        for (int r = threadIdx.x; r < HB * HB * HB; r += blockDim.x) c = fmaxf(c, (float)nh[r]);
        c = warp_max(c);
        const float a = warp_max(nu2), b = warp_max(nwm);
        if (lane == 0) { s_max[0][wid] = a; s_max[1][wid] = b; s_max[2][wid] = c; }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < nwarps; ++w) t += s_red[w];
        sj.ke_tile[tile] = t * sj.m * sj.clight * sj.clight;
        if (FIXED && stats) {
          float a = 0.f, b = 0.f, c = 0.f;
          for (int w = 0; w < nwarps; ++w) {
            a = fmaxf(a, s_max[0][w]); b = fmaxf(b, s_max[1][w]); c = fmaxf(c, s_max[2][w]);
          }
          stats[0] = a; stats[1] = b; stats[2] = c; stats[3] = 1.f;
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace pxrt
