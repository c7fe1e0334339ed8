// Tiled engine: the B200-native per-step particle loop.
//
// Layout (see pxrb_tiled_job in picsar_b200.h): E/B in the engine precision R
// (float or double) with g periodic guard cells, J in FP64 without guards,
// particles sorted by cell tile as (packed cell, in-cell offset, u, w).
//
// One fused kernel per step does, for every tile: stage the tile's E/B window
// in shared memory, gather + push + position update + periodic wrap for each
// particle of the tile, and Esirkepov deposition from the exact old position
// into a shared-memory J window, flushed once to the global FP64 J with
// atomics.  Particles that drifted out of the tile window since the last sort
// use the global-memory path (same arithmetic, global loads/atomics).
//
// Formulas: gather/push particle_pusher_manager_3d.F90:1287-2193 (energy
// conserving, l_lower_order_in_v), Boris boris_3d.F90:96-131 + set_gamma,
// Vay vay_3d.F90:100-130, Esirkepov esirkepov_3d.F90:82-239, :1734-1918,
// :3263-3464, Yee yee.F90:637-740, :1258-1347.
#include "pxr_common.cuh"
#include "picsar_b200.h"

#include <cub/block/block_scan.cuh>

namespace {

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

// Shared-memory accumulator type: FP32 window for the mixed engine, FP64 for
// the FP64 engine.
template <typename R> struct AccT { typedef R type; };

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

template <typename R> __device__ __forceinline__ R rsqrt_(R x);
template <> __device__ __forceinline__ float rsqrt_<float>(float x) { return 1.0f / sqrtf(x); }
template <> __device__ __forceinline__ double rsqrt_<double>(double x) { return 1.0 / sqrt(x); }

constexpr int MAX_THREADS = 256;

// ---------------------------------------------------------------------------
// The fused particle kernel (persistent CTAs pulling (job, tile) items).
// ---------------------------------------------------------------------------
template <typename R, int ORDER>
__global__ void __launch_bounds__(MAX_THREADS)
    k_tiled_step(const Job* __restrict__ jobs, const int2* __restrict__ work, int nwork,
                 const int* __restrict__ nwork_dev, int* ctr) {
  typedef typename AccT<R>::type A;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ Job sj;
  __shared__ int s_item;
  __shared__ double s_red[MAX_THREADS / 32];
  constexpr int L = Reach<ORDER>::L, H = Reach<ORDER>::H;

  if (nwork_dev) nwork = min(nwork, *nwork_dev);
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(ctr, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nwork) break;
    const int2 wk = work[item];
    // job descriptor into shared memory
    {
      const int nw = (int)(sizeof(Job) / sizeof(int));
      const int* src = reinterpret_cast<const int*>(jobs + wk.x);
      int* dst = reinterpret_cast<int*>(&sj);
      for (int t = threadIdx.x; t < nw; t += blockDim.x) dst[t] = src[t];
    }
    __syncthreads();
    const int nx = sj.nx, ny = sj.ny, nz = sj.nz, G = sj.g, D = sj.drift;
    const int tile = wk.y;
    const int ti = tile % sj.ntx, tj = (tile / sj.ntx) % sj.nty, tk = tile / (sj.ntx * sj.nty);
    const int c0x = ti * sj.tx, c0y = tj * sj.ty, c0z = tk * sj.tz;
    const int tex = min(sj.tx, nx - c0x), tey = min(sj.ty, ny - c0y), tez = min(sj.tz, nz - c0z);
    const int Wx = tex + 2 * D + L + H, Wy = tey + 2 * D + L + H, Wz = tez + 2 * D + L + H;
    const int wox = c0x - D - L, woy = c0y - D - L, woz = c0z - D - L;
    const int V = Wx * Wy * Wz;
    R* Fs = reinterpret_cast<R*>(smem_raw);
    A* Js = reinterpret_cast<A*>(smem_raw + (size_t)6 * V * sizeof(R));
    // ---- stage E/B window (guarded global arrays: no wrap needed) -------
    const int pitch = sj.pitch_x, NYg = ny + 2 * G;
    const R* gF[6] = {(const R*)sj.ex, (const R*)sj.ey, (const R*)sj.ez,
                      (const R*)sj.bx, (const R*)sj.by, (const R*)sj.bz};
    for (int e = threadIdx.x; e < 6 * V; e += blockDim.x) {
      int comp = e / V, r = e - comp * V;
      int a = r % Wx, rb = r / Wx, b = rb % Wy, c = rb / Wy;
      i64 gidx = (i64)(wox + a + G) + (i64)pitch * ((woy + b + G) + (i64)NYg * (woz + c + G));
      Fs[e] = __ldg(gF[comp] + gidx);
    }
    for (int e = threadIdx.x; e < 3 * V; e += blockDim.x) Js[e] = (A)0;
    __syncthreads();

    FieldView<R> FW[6], FG[6];
    for (int c = 0; c < 6; ++c) {
      FW[c].p = Fs + c * V; FW[c].sy = Wx; FW[c].sz = Wx * Wy;
      FG[c].p = gF[c] + (G + (i64)pitch * (G + (i64)NYg * G));
      FG[c].sy = pitch; FG[c].sz = pitch * NYg;
    }
    SmemAcc<A> JW[3];
    for (int c = 0; c < 3; ++c) { JW[c].p = Js + c * V; JW[c].sy = Wx; JW[c].sz = Wx * Wy; }
    GlobAcc JG[3];
    JG[0].p = sj.jx; JG[1].p = sj.jy; JG[2].p = sj.jz;
    for (int c = 0; c < 3; ++c) { JG[c].nx = nx; JG[c].ny = ny; JG[c].nz = nz; }

    const R dtdx = (R)(sj.dt / sj.dx), dtdy = (R)(sj.dt / sj.dy), dtdz = (R)(sj.dt / sj.dz);
    const R clghtisq = (R)(1.0 / (sj.clight * sj.clight));
    const R cst_b = (R)(sj.q * sj.dt * 0.5 / sj.m), cst_v = (R)(sj.q * sj.dt / sj.m);
    const R invc = (R)(1.0 / sj.clight);
    const double invdtdx = 1.0 / (sj.dt * sj.dy * sj.dz), invdtdy = 1.0 / (sj.dt * sj.dx * sj.dz),
                 invdtdz = 1.0 / (sj.dt * sj.dx * sj.dy);
    const bool vay = sj.pusher == 1;
    uint32_t* cellp = sj.cell;
    R *oxp = (R*)sj.ox, *oyp = (R*)sj.oy, *ozp = (R*)sj.oz;
    R *uxp = (R*)sj.ux, *uyp = (R*)sj.uy, *uzp = (R*)sj.uz;
    const R* wp = (const R*)sj.w;
    const int pbeg = sj.tile_off[tile], pend = sj.tile_off[tile + 1];
    double ke = 0.0;
    int nslow = 0, bad = 0;

    for (int ip = pbeg + threadIdx.x; ip < pend; ip += blockDim.x) {
      int ci, cj, ck;
      unpack_cell(cellp[ip], ci, cj, ck);
      R ox = oxp[ip], oy = oyp[ip], oz = ozp[ip];
      R ux = uxp[ip], uy = uyp[ip], uz = uzp[ip];
      const R wgt = wp[ip];
      // tile-relative cell, unwrapped to the nearest periodic image
      int vx = ci - c0x, vy = cj - c0y, vz = ck - c0z;
      if (vx > tex - 1 + D) vx -= nx; else if (vx < -D) vx += nx;
      if (vy > tey - 1 + D) vy -= ny; else if (vy < -D) vy += ny;
      if (vz > tez - 1 + D) vz -= nz; else if (vz < -D) vz += nz;
      const bool in_old = vx >= -D && vx <= tex - 1 + D && vy >= -D && vy <= tey - 1 + D &&
                          vz >= -D && vz <= tez - 1 + D;
      // ---- gather ----------------------------------------------------------
      R eb[6];
      if (in_old) {
        gather6<ORDER, R>(FW, vx + D + L, vy + D + L, vz + D + L, ox, oy, oz, eb);
      } else {
        gather6<ORDER, R>(FG, ci, cj, ck, ox, oy, oz, eb);
      }
      // ---- push ------------------------------------------------------------
      R gi;
      if (vay) {
        gi = rsqrt_<R>((R)1 + (ux * ux + uy * uy + uz * uz) * clghtisq);
        vay_push(ux, uy, uz, gi, eb[0], eb[1], eb[2], eb[3], eb[4], eb[5], cst_v, invc, clghtisq);
      } else {
        boris_push(ux, uy, uz, gi, eb[0], eb[1], eb[2], eb[3], eb[4], eb[5], cst_b, clghtisq);
        set_gamma(ux, uy, uz, gi, clghtisq);
      }
      // ---- position: exact old (c, o), new (c', o') -------------------------
      R nox = ox, noy = oy, noz = oz;
      int ncx = 0, ncy = 0, ncz = 0;   // cell shift
      cell_step(nox, ncx, ux * gi * dtdx);
      cell_step(noy, ncy, uy * gi * dtdy);
      cell_step(noz, ncz, uz * gi * dtdz);
      // ---- deposition ------------------------------------------------------
      int r0, r1;
      R xi0, xi1;
      EsirAxis<ORDER, R> EX, EY, EZ;
      bool ok = true;
      const R wq = (R)(sj.q) * wgt;
      const R wqx = wq * (R)invdtdx, wqy = wq * (R)invdtdy, wqz = wq * (R)invdtdz;
      const bool in_new = in_old && vx + ncx >= -D && vx + ncx <= tex - 1 + D &&
                          vy + ncy >= -D && vy + ncy <= tey - 1 + D && vz + ncz >= -D &&
                          vz + ncz <= tez - 1 + D;
      // cell coordinates of the old position in the accumulator's frame
      const int bx = in_new ? vx + D + L : ci;
      const int by = in_new ? vy + D + L : cj;
      const int bz = in_new ? vz + D + L : ck;
      esir_node<ORDER, R>(nox, r0, xi0);
      esir_node<ORDER, R>(ox, r1, xi1);
      ok = EX.set(bx + ncx + r0, xi0, bx + r1, xi1) && ok;
      esir_node<ORDER, R>(noy, r0, xi0);
      esir_node<ORDER, R>(oy, r1, xi1);
      ok = EY.set(by + ncy + r0, xi0, by + r1, xi1) && ok;
      esir_node<ORDER, R>(noz, r0, xi0);
      esir_node<ORDER, R>(oz, r1, xi1);
      ok = EZ.set(bz + ncz + r0, xi0, bz + r1, xi1) && ok;
      if (!ok) bad = 1;
      if (in_new) {
        esirkepov_dep<ORDER, R, SmemAcc<A>, A>(EX, EY, EZ, wqx, wqy, wqz, JW[0], JW[1], JW[2]);
      } else {
        ++nslow;
        esirkepov_dep<ORDER, R, GlobAcc, double>(EX, EY, EZ, wqx, wqy, wqz, JG[0], JG[1], JG[2]);
      }
      // ---- store -----------------------------------------------------------
      int nci = ci + ncx, ncj = cj + ncy, nck = ck + ncz;
      nci = nci < 0 ? nci + nx : (nci >= nx ? nci - nx : nci);
      ncj = ncj < 0 ? ncj + ny : (ncj >= ny ? ncj - ny : ncj);
      nck = nck < 0 ? nck + nz : (nck >= nz ? nck - nz : nck);
      cellp[ip] = pack_cell(nci, ncj, nck);
      oxp[ip] = nox; oyp[ip] = noy; ozp[ip] = noz;
      uxp[ip] = ux; uyp[ip] = uy; uzp[ip] = uz;
      // kinetic energy (gamma - 1) w, in FP64 from u
      const double u2 = (double)ux * ux + (double)uy * uy + (double)uz * uz;
      const double c2i = 1.0 / (sj.clight * sj.clight);
      ke += u2 * c2i / (1.0 + sqrt(1.0 + u2 * c2i)) * (double)wgt;
    }
    __syncthreads();
    // ---- flush J window (FP64 atomics, zeros skipped) ----------------------
    {
      double* gJ[3] = {sj.jx, sj.jy, sj.jz};
      for (int e = threadIdx.x; e < 3 * V; e += blockDim.x) {
        A v = Js[e];
        if (v == (A)0) continue;
        int comp = e / V, r = e - comp * V;
        int a = r % Wx, rb = r / Wx, b = rb % Wy, c = rb / Wy;
        int gi = GlobAcc::wrap(wox + a, nx), gj = GlobAcc::wrap(woy + b, ny),
            gk = GlobAcc::wrap(woz + c, nz);
        atomicAdd(gJ[comp] + gi + (i64)nx * (gj + (i64)ny * gk), (double)v);
      }
    }
    // ---- kinetic energy of the tile (deterministic per-tile partial) -------
    {
      double v = ke;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
      // counters
      if (nslow) atomicAdd(&sj.counters[0], nslow);
      if (bad) atomicExch(&sj.counters[1], 1);
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_red[w];
        sj.ke_tile[tile] = t * sj.m * sj.clight * sj.clight;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Yee on the guarded engine layout, all jobs in one launch.  Thread = cell.
// cell_off[j]: start of job j in the flat cell index space (multiple of the
// block size).  Writes the periodic images of each updated value into the
// guard cells.
// ---------------------------------------------------------------------------
constexpr int YEE_TPB = 256;

__device__ __forceinline__ int find_job(const int64_t* off, int njobs, int64_t gid) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= gid) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename R>
__device__ __forceinline__ void store_images(R* base, int i, int j, int k, int nx, int ny,
                                             int nz, int G, int pitch, int NYg, R v) {
  int ii[2] = {i, 0}, jj[2] = {j, 0}, kk[2] = {k, 0};
  int ni = 1, nj = 1, nk = 1;
  if (i < G) ii[ni++] = i + nx; else if (i >= nx - G) ii[ni++] = i - nx;
  if (j < G) jj[nj++] = j + ny; else if (j >= ny - G) jj[nj++] = j - ny;
  if (k < G) kk[nk++] = k + nz; else if (k >= nz - G) kk[nk++] = k - nz;
  for (int c = 0; c < nk; ++c)
    for (int b = 0; b < nj; ++b)
      for (int a = 0; a < ni; ++a)
        base[(ii[a] + G) + (i64)pitch * ((jj[b] + G) + (i64)NYg * (kk[c] + G))] = v;
}

template <typename R>
__global__ void __launch_bounds__(YEE_TPB)
    k_yee_b_t(const Job* __restrict__ jobs, int njobs, const int64_t* __restrict__ off, R frac) {
  __shared__ int s_job;
  const int64_t gid0 = (int64_t)blockIdx.x * YEE_TPB;
  if (threadIdx.x == 0) s_job = find_job(off, njobs, gid0);
  __syncthreads();
  const Job& J = jobs[s_job];
  const int64_t lid = gid0 - off[s_job] + threadIdx.x;
  const int nx = J.nx, ny = J.ny, nz = J.nz;
  if (lid >= (int64_t)nx * ny * nz) return;
  const int i = (int)(lid % nx), j = (int)((lid / nx) % ny), k = (int)(lid / ((int64_t)nx * ny));
  const int G = J.g, pitch = J.pitch_x, NYg = ny + 2 * G;
  const i64 sy = pitch, sz = (i64)pitch * NYg;
  const i64 c = (i + G) + sy * (j + G) + sz * (k + G);
  const R* ex = (const R*)J.ex; const R* ey = (const R*)J.ey; const R* ez = (const R*)J.ez;
  R* bx = (R*)J.bx; R* by = (R*)J.by; R* bz = (R*)J.bz;
  const R dtsdx = (R)(frac * J.dt / J.dx), dtsdy = (R)(frac * J.dt / J.dy),
          dtsdz = (R)(frac * J.dt / J.dz);
  const R ezc = ez[c], eyc = ey[c], exc = ex[c];
  R vbx = bx[c] - dtsdy * (ez[c + sy] - ezc) + dtsdz * (ey[c + sz] - eyc);
  R vby = by[c] + dtsdx * (ez[c + 1] - ezc) - dtsdz * (ex[c + sz] - exc);
  R vbz = bz[c] - dtsdx * (ey[c + 1] - eyc) + dtsdy * (ex[c + sy] - exc);
  store_images(bx, i, j, k, nx, ny, nz, G, pitch, NYg, vbx);
  store_images(by, i, j, k, nx, ny, nz, G, pitch, NYg, vby);
  store_images(bz, i, j, k, nx, ny, nz, G, pitch, NYg, vbz);
}

template <typename R>
__global__ void __launch_bounds__(YEE_TPB)
    k_yee_e_t(const Job* __restrict__ jobs, int njobs, const int64_t* __restrict__ off,
              int zero_j) {
  __shared__ int s_job;
  const int64_t gid0 = (int64_t)blockIdx.x * YEE_TPB;
  if (threadIdx.x == 0) s_job = find_job(off, njobs, gid0);
  __syncthreads();
  const Job& J = jobs[s_job];
  const int64_t lid = gid0 - off[s_job] + threadIdx.x;
  const int nx = J.nx, ny = J.ny, nz = J.nz;
  if (lid >= (int64_t)nx * ny * nz) return;
  const int i = (int)(lid % nx), j = (int)((lid / nx) % ny), k = (int)(lid / ((int64_t)nx * ny));
  const int G = J.g, pitch = J.pitch_x, NYg = ny + 2 * G;
  const i64 sy = pitch, sz = (i64)pitch * NYg;
  const i64 c = (i + G) + sy * (j + G) + sz * (k + G);
  R* ex = (R*)J.ex; R* ey = (R*)J.ey; R* ez = (R*)J.ez;
  const R* bx = (const R*)J.bx; const R* by = (const R*)J.by; const R* bz = (const R*)J.bz;
  const double c2 = J.clight * J.clight;
  const R mudt = (R)(c2 * J.mu0 * J.dt), dtsdx = (R)(c2 * J.dt / J.dx),
          dtsdy = (R)(c2 * J.dt / J.dy), dtsdz = (R)(c2 * J.dt / J.dz);
  const i64 jc = lid;
  const R jxv = (R)J.jx[jc], jyv = (R)J.jy[jc], jzv = (R)J.jz[jc];
  if (zero_j) { J.jx[jc] = 0.0; J.jy[jc] = 0.0; J.jz[jc] = 0.0; }
  const R bzc = bz[c], byc = by[c], bxc = bx[c];
  R vex = ex[c] + dtsdy * (bzc - bz[c - sy]) - dtsdz * (byc - by[c - sz]) - mudt * jxv;
  R vey = ey[c] - dtsdx * (bzc - bz[c - 1]) + dtsdz * (bxc - bx[c - sz]) - mudt * jyv;
  R vez = ez[c] + dtsdx * (byc - by[c - 1]) - dtsdy * (bxc - bx[c - sy]) - mudt * jzv;
  store_images(ex, i, j, k, nx, ny, nz, G, pitch, NYg, vex);
  store_images(ey, i, j, k, nx, ny, nz, G, pitch, NYg, vey);
  store_images(ez, i, j, k, nx, ny, nz, G, pitch, NYg, vez);
}

// ---------------------------------------------------------------------------
// Counting sort by tile.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int tile_of(const Job& J, uint32_t cell) {
  int i, j, k;
  unpack_cell(cell, i, j, k);
  return i / J.tx + J.ntx * (j / J.ty + J.nty * (k / J.tz));
}

__global__ void k_sort_count(const Job* __restrict__ jp) {
  const Job& J = *jp;
  const int ntiles = J.ntx * J.nty * J.ntz;
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < J.np;
       p += (i64)gridDim.x * blockDim.x) {
    int t = tile_of(J, J.cell[p]);
    // aggregate equal tiles inside the warp
    unsigned mask = __activemask();
    unsigned peers = __match_any_sync(mask, t);
    int leader = __ffs(peers) - 1;
    if ((threadIdx.x & 31) == leader) atomicAdd(&J.tile_cnt[t], __popc(peers));
    (void)ntiles;
  }
}

constexpr int SCAN_TPB = 1024;

// exclusive scan of tile_cnt into tile_off, cursor copy left in tile_cnt
__global__ void __launch_bounds__(SCAN_TPB) k_sort_scan(const Job* __restrict__ jp) {
  typedef cub::BlockScan<int, SCAN_TPB> Scan;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ int carry;
  const Job& J = *jp;
  const int ntiles = J.ntx * J.nty * J.ntz;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < ntiles; base += SCAN_TPB) {
    int t = base + threadIdx.x;
    int v = t < ntiles ? J.tile_cnt[t] : 0;
    int ex, tot;
    Scan(tmp).ExclusiveSum(v, ex, tot);
    int c0 = carry;
    if (t < ntiles) { J.tile_off[t] = c0 + ex; J.tile_cnt[t] = c0 + ex; }
    __syncthreads();
    if (threadIdx.x == 0) carry = c0 + tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) J.tile_off[ntiles] = carry;
}

template <typename R>
__global__ void k_sort_scatter(const Job* __restrict__ jp) {
  const Job& J = *jp;
  const R *ox = (const R*)J.ox, *oy = (const R*)J.oy, *oz = (const R*)J.oz;
  const R *ux = (const R*)J.ux, *uy = (const R*)J.uy, *uz = (const R*)J.uz, *w = (const R*)J.w;
  R *ox2 = (R*)J.ox_b, *oy2 = (R*)J.oy_b, *oz2 = (R*)J.oz_b;
  R *ux2 = (R*)J.ux_b, *uy2 = (R*)J.uy_b, *uz2 = (R*)J.uz_b, *w2 = (R*)J.w_b;
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < J.np;
       p += (i64)gridDim.x * blockDim.x) {
    uint32_t cell = J.cell[p];
    int t = tile_of(J, cell);
    unsigned mask = __activemask();
    unsigned peers = __match_any_sync(mask, t);
    int lane = threadIdx.x & 31;
    int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&J.tile_cnt[t], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    int slot = base + __popc(peers & ((1u << lane) - 1u));
    J.cell_b[slot] = cell;
    ox2[slot] = ox[p]; oy2[slot] = oy[p]; oz2[slot] = oz[p];
    ux2[slot] = ux[p]; uy2[slot] = uy[p]; uz2[slot] = uz[p]; w2[slot] = w[p];
    if (J.pid) J.pid_b[slot] = J.pid[p];
  }
}

// swap the particle arrays with the sort buffers in the device descriptor
__global__ void k_sort_swap(Job* jp) {
  Job& J = *jp;
  uint32_t* c = J.cell; J.cell = J.cell_b; J.cell_b = c;
  void* t;
  t = J.ox; J.ox = J.ox_b; J.ox_b = t;
  t = J.oy; J.oy = J.oy_b; J.oy_b = t;
  t = J.oz; J.oz = J.oz_b; J.oz_b = t;
  t = J.ux; J.ux = J.ux_b; J.ux_b = t;
  t = J.uy; J.uy = J.uy_b; J.uy_b = t;
  t = J.uz; J.uz = J.uz_b; J.uz_b = t;
  t = J.w; J.w = J.w_b; J.w_b = t;
  int32_t* q = J.pid; J.pid = J.pid_b; J.pid_b = q;
}

// ---------------------------------------------------------------------------
// Conversions
// ---------------------------------------------------------------------------
template <typename R>
__global__ void k_load_particles(Job J, const double* x, const double* y, const double* z,
                                 const double* ux, const double* uy, const double* uz,
                                 const double* w) {
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < J.np;
       p += (i64)gridDim.x * blockDim.x) {
    double pos[3] = {(x[p] - J.xmin) / J.dx, (y[p] - J.ymin) / J.dy, (z[p] - J.zmin) / J.dz};
    int n[3] = {J.nx, J.ny, J.nz};
    int c[3];
    R o[3];
    for (int a = 0; a < 3; ++a) {
      double f = floor(pos[a]);
      int ci = (int)f;
      R oo = (R)(pos[a] - f);
      if (oo >= (R)1) { oo = (R)0; ci += 1; }
      ci %= n[a];
      if (ci < 0) ci += n[a];
      c[a] = ci; o[a] = oo;
    }
    J.cell[p] = pack_cell(c[0], c[1], c[2]);
    ((R*)J.ox)[p] = o[0]; ((R*)J.oy)[p] = o[1]; ((R*)J.oz)[p] = o[2];
    ((R*)J.ux)[p] = (R)ux[p]; ((R*)J.uy)[p] = (R)uy[p]; ((R*)J.uz)[p] = (R)uz[p];
    ((R*)J.w)[p] = (R)w[p];
  }
}

template <typename R>
__global__ void k_store_particles(Job J, double* x, double* y, double* z, double* ux,
                                  double* uy, double* uz, double* gaminv, double* w) {
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < J.np;
       p += (i64)gridDim.x * blockDim.x) {
    int i, j, k;
    unpack_cell(J.cell[p], i, j, k);
    if (x) x[p] = J.xmin + ((double)i + (double)((const R*)J.ox)[p]) * J.dx;
    if (y) y[p] = J.ymin + ((double)j + (double)((const R*)J.oy)[p]) * J.dy;
    if (z) z[p] = J.zmin + ((double)k + (double)((const R*)J.oz)[p]) * J.dz;
    double a = ((const R*)J.ux)[p], b = ((const R*)J.uy)[p], c = ((const R*)J.uz)[p];
    if (ux) ux[p] = a;
    if (uy) uy[p] = b;
    if (uz) uz[p] = c;
    if (gaminv) gaminv[p] = 1.0 / sqrt(1.0 + (a * a + b * b + c * c) / (J.clight * J.clight));
    if (w) w[p] = ((const R*)J.w)[p];
  }
}

// Fortran guarded FP64 grid (ng guards) <-> engine.  dir 0: import, 1: export.
template <typename R>
__global__ void k_field_xfer(Job J, int which, double* f, int ng, int dir) {
  const int nx = J.nx, ny = J.ny, nz = J.nz, G = J.g;
  if (which < 6) {
    R* e = (R*)((&J.ex)[which]);
    const int ex_ = nx + 2 * G, ey_ = ny + 2 * G, ez_ = nz + 2 * G;
    const i64 total = (i64)ex_ * ey_ * ez_;
    const int sx = nx + 1 + 2 * ng, sy = ny + 1 + 2 * ng;
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total;
         t += (i64)gridDim.x * blockDim.x) {
      int a = (int)(t % ex_), b = (int)((t / ex_) % ey_), c = (int)(t / ((i64)ex_ * ey_));
      int i = a - G, j = b - G, k = c - G;
      int pi = ((i % nx) + nx) % nx, pj = ((j % ny) + ny) % ny, pk = ((k % nz) + nz) % nz;
      i64 e_idx = a + (i64)J.pitch_x * (b + (i64)ey_ * c);
      if (dir == 0) {
        e[e_idx] = (R)f[(pi + ng) + (i64)sx * ((pj + ng) + (i64)sy * (pk + ng))];
      } else if (i >= -ng && i <= nx + ng && j >= -ng && j <= ny + ng && k >= -ng &&
                 k <= nz + ng) {
        f[(i + ng) + (i64)sx * ((j + ng) + (i64)sy * (k + ng))] = (double)e[e_idx];
      }
    }
    if (dir == 1) {
      // nodes beyond the engine guards (ng > G) get periodic images
      const i64 tot2 = (i64)(nx + 1 + 2 * ng) * (ny + 1 + 2 * ng) * (nz + 1 + 2 * ng);
      for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < tot2;
           t += (i64)gridDim.x * blockDim.x) {
        int a = (int)(t % sx), b = (int)((t / sx) % sy), c = (int)(t / ((i64)sx * sy));
        int i = a - ng, j = b - ng, k = c - ng;
        if (i >= -G && i < nx + G && j >= -G && j < ny + G && k >= -G && k < nz + G) continue;
        int pi = ((i % nx) + nx) % nx, pj = ((j % ny) + ny) % ny, pk = ((k % nz) + nz) % nz;
        f[t] = (double)e[(pi + G) + (i64)J.pitch_x * ((pj + G) + (i64)ey_ * (pk + G))];
      }
    }
  } else {
    double* jj = (&J.jx)[which - 6];
    const int sx = nx + 1 + 2 * ng, sy = ny + 1 + 2 * ng;
    const i64 total = dir == 0 ? (i64)nx * ny * nz : (i64)sx * sy * (nz + 1 + 2 * ng);
    for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total;
         t += (i64)gridDim.x * blockDim.x) {
      if (dir == 0) {
        int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / ((i64)nx * ny));
        jj[t] = f[(i + ng) + (i64)sx * ((j + ng) + (i64)sy * (k + ng))];
      } else {
        int a = (int)(t % sx), b = (int)((t / sx) % sy), c = (int)(t / ((i64)sx * sy));
        int i = a - ng, j = b - ng, k = c - ng;
        int pi = ((i % nx) + nx) % nx, pj = ((j % ny) + ny) % ny, pk = ((k % nz) + nz) % nz;
        f[t] = jj[pi + (i64)nx * (pj + (i64)ny * pk)];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Diagnostics
// ---------------------------------------------------------------------------
template <typename R, int ORDER>
__global__ void k_rho_t(Job J, double* rho) {
  for (i64 p = blockIdx.x * (i64)blockDim.x + threadIdx.x; p < J.np;
       p += (i64)gridDim.x * blockDim.x) {
    int ci, cj, ck;
    unpack_cell(J.cell[p], ci, cj, ck);
    NodeCO<ORDER, double> sx, sy, sz;
    sx.set((double)((const R*)J.ox)[p]);
    sy.set((double)((const R*)J.oy)[p]);
    sz.set((double)((const R*)J.oz)[p]);
    const double wq = J.q * (double)((const R*)J.w)[p] / (J.dx * J.dy * J.dz);
#pragma unroll
    for (int c = 0; c < ORDER + 1; ++c)
#pragma unroll
      for (int b = 0; b < ORDER + 1; ++b)
#pragma unroll
        for (int a = 0; a < ORDER + 1; ++a) {
          int i = GlobAcc::wrap(ci + sx.r0 + a, J.nx), j = GlobAcc::wrap(cj + sy.r0 + b, J.ny),
              k = GlobAcc::wrap(ck + sz.r0 + c, J.nz);
          atomicAdd(rho + i + (i64)J.nx * (j + (i64)J.ny * k), sx.s[a] * sy.s[b] * sz.s[c] * wq);
        }
  }
}

constexpr int RED_TPB = 256;

// per-block partial sums: [0..5] 0.5 F^2 of the six fields, [6] (divE eps0 - rho)^2,
// [7] rho^2; part[q * nblocks + block]
template <typename R>
__global__ void __launch_bounds__(RED_TPB) k_field_sums(Job J, const double* rho, double* part) {
  const int nx = J.nx, ny = J.ny, nz = J.nz, G = J.g, pitch = J.pitch_x, NYg = ny + 2 * G;
  const i64 sy = pitch, sz = (i64)pitch * NYg;
  const i64 total = (i64)nx * ny * nz;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const R* F[6] = {(const R*)J.ex, (const R*)J.ey, (const R*)J.ez,
                   (const R*)J.bx, (const R*)J.by, (const R*)J.bz};
  for (i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x; t < total;
       t += (i64)gridDim.x * blockDim.x) {
    int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / ((i64)nx * ny));
    i64 c = (i + G) + sy * (j + G) + sz * (k + G);
    for (int q = 0; q < 6; ++q) {
      double v = (double)F[q][c];
      acc[q] += v * v * 0.5;
    }
    if (rho) {
      double dive = ((double)F[0][c] - (double)F[0][c - 1]) / J.dx +
                    ((double)F[1][c] - (double)F[1][c - sy]) / J.dy +
                    ((double)F[2][c] - (double)F[2][c - sz]) / J.dz;
      double r = rho[t];
      double d = dive * J.eps0 - r;
      acc[6] += d * d;
      acc[7] += r * r;
    }
  }
  __shared__ double red[8][RED_TPB / 32];
  for (int q = 0; q < 8; ++q) {
    double v = acc[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double s = 0;
    for (int w = 0; w < RED_TPB / 32; ++w) s += red[threadIdx.x][w];
    part[threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void k_diag_final(Job J, const double* part, int nblocks, double* out) {
  // one warp; fixed order
  __shared__ double s[9];
  if (threadIdx.x < 8) {
    double t = 0;
    for (int b = 0; b < nblocks; ++b) t += part[threadIdx.x * nblocks + b];
    s[threadIdx.x] = t;
  }
  if (threadIdx.x == 8) {
    double t = 0;
    const int ntiles = J.ntx * J.nty * J.ntz;
    for (int b = 0; b < ntiles; ++b) t += J.ke_tile[b];
    s[8] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double dv = J.dx * J.dy * J.dz;
    out[0] = s[8];
    for (int q = 0; q < 3; ++q) out[1 + q] = s[q] * dv * J.eps0;
    for (int q = 3; q < 6; ++q) out[1 + q] = s[q] * dv / J.mu0;
    out[7] = sqrt(s[6]);
    out[8] = sqrt(s[7]);
  }
}

int diag_blocks(const Job& J) {
  i64 total = (i64)J.nx * J.ny * J.nz;
  i64 b = (total + RED_TPB - 1) / RED_TPB;
  return (int)(b > 1184 ? 1184 : (b < 1 ? 1 : b));
}

template <int ORDER>
constexpr int reach_total() { return Reach<ORDER>::L + Reach<ORDER>::H; }

int64_t smem_bytes(int order, int prec, int tx, int ty, int tz, int drift) {
  int lh = order == 1 ? 1 : 3;
  i64 V = (i64)(tx + 2 * drift + lh) * (ty + 2 * drift + lh) * (tz + 2 * drift + lh);
  i64 r = prec ? 8 : 4;
  return V * (6 * r + 3 * r);
}

template <typename R, int ORDER>
int launch_step(const Job* jobs, const int2* work, int nwork, const int* nwork_dev, int* ctr,
                int threads, int ctas, size_t smem, cudaStream_t s) {
  auto kern = k_tiled_step<R, ORDER>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return PXRB_EUNSUPPORTED;
  if (cudaMemsetAsync(ctr, 0, sizeof(int), s) != cudaSuccess) return PXRB_ELAUNCH;
  kern<<<ctas, threads, smem, s>>>(jobs, work, nwork, nwork_dev, ctr);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

inline int gs_blocks(i64 n, int tpb) {
  i64 b = (n + tpb - 1) / tpb;
  const i64 cap = 148 * 32;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

extern "C" {

int64_t pxrb_tiled_job_size(void) { return (int64_t)sizeof(pxrb_tiled_job); }

int64_t pxrb_tiled_smem_bytes(int32_t order, int32_t prec, int32_t tx, int32_t ty, int32_t tz,
                              int32_t drift) {
  return smem_bytes(order, prec, tx, ty, tz, drift);
}

int pxrb_tiled_particle_step(const pxrb_tiled_job* jobs_dev, int32_t order, int32_t prec,
                             const int32_t* work, int32_t nwork, const int32_t* nwork_dev,
                             int32_t* ctr, int32_t threads, int32_t ctas, int64_t smem,
                             void* stream) {
  if (!jobs_dev || !work || !ctr || nwork < 0 || smem < 0) return PXRB_EINVAL;
  if (nwork == 0) return PXRB_OK;
  if (threads < 32 || threads > MAX_THREADS || threads % 32) return PXRB_EINVAL;
  if (order < 1 || order > 3 || prec < 0 || prec > 1) return PXRB_EUNSUPPORTED;
  if (ctas < 1) ctas = 1;
  cudaStream_t s = (cudaStream_t)stream;
  const int2* w2 = reinterpret_cast<const int2*>(work);
#define PXRB_STEP(R_, O_) \
  return launch_step<R_, O_>(jobs_dev, w2, nwork, nwork_dev, ctr, threads, ctas, (size_t)smem, s);
  if (prec == 0) {
    if (order == 1) { PXRB_STEP(float, 1) }
    if (order == 2) { PXRB_STEP(float, 2) }
    PXRB_STEP(float, 3)
  } else {
    if (order == 1) { PXRB_STEP(double, 1) }
    if (order == 2) { PXRB_STEP(double, 2) }
    PXRB_STEP(double, 3)
  }
#undef PXRB_STEP
}

int pxrb_tiled_push_b(const pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                      const int64_t* cell_off_dev, int64_t total_cells, double frac,
                      void* stream) {
  if (!jobs_dev || !cell_off_dev || njobs < 1 || total_cells < 0) return PXRB_EINVAL;
  if (total_cells == 0) return PXRB_OK;
  int nb = (int)((total_cells + YEE_TPB - 1) / YEE_TPB);
  cudaStream_t s = (cudaStream_t)stream;
  if (prec == 0) k_yee_b_t<float><<<nb, YEE_TPB, 0, s>>>(jobs_dev, njobs, cell_off_dev, (float)frac);
  else k_yee_b_t<double><<<nb, YEE_TPB, 0, s>>>(jobs_dev, njobs, cell_off_dev, frac);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_push_e(const pxrb_tiled_job* jobs_dev, int32_t njobs, int32_t prec,
                      const int64_t* cell_off_dev, int64_t total_cells, int32_t zero_j,
                      void* stream) {
  if (!jobs_dev || !cell_off_dev || njobs < 1 || total_cells < 0) return PXRB_EINVAL;
  if (total_cells == 0) return PXRB_OK;
  int nb = (int)((total_cells + YEE_TPB - 1) / YEE_TPB);
  cudaStream_t s = (cudaStream_t)stream;
  if (prec == 0) k_yee_e_t<float><<<nb, YEE_TPB, 0, s>>>(jobs_dev, njobs, cell_off_dev, zero_j);
  else k_yee_e_t<double><<<nb, YEE_TPB, 0, s>>>(jobs_dev, njobs, cell_off_dev, zero_j);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_sort(const pxrb_tiled_job* job_host, pxrb_tiled_job* job_dev, void* stream) {
  if (!job_host || !job_dev) return PXRB_EINVAL;
  const Job& J = *job_host;
  if (J.np < 0 || !J.tile_cnt || !J.tile_off) return PXRB_EINVAL;
  const int ntiles = J.ntx * J.nty * J.ntz;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(J.tile_cnt, 0, sizeof(int32_t) * (ntiles + 1), s) != cudaSuccess)
    return PXRB_ELAUNCH;
  const int nb = gs_blocks(J.np, 256);
  if (J.np > 0) k_sort_count<<<nb, 256, 0, s>>>(job_dev);
  k_sort_scan<<<1, SCAN_TPB, 0, s>>>(job_dev);
  if (J.np > 0) {
    if (J.prec == 0) k_sort_scatter<float><<<nb, 256, 0, s>>>(job_dev);
    else k_sort_scatter<double><<<nb, 256, 0, s>>>(job_dev);
    k_sort_swap<<<1, 1, 0, s>>>(job_dev);
  }
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_load_particles(const pxrb_tiled_job* job_host, const double* x, const double* y,
                              const double* z, const double* ux, const double* uy,
                              const double* uz, const double* w, void* stream) {
  if (!job_host) return PXRB_EINVAL;
  const Job& J = *job_host;
  if (J.np == 0) return PXRB_OK;
  if (!x || !y || !z || !ux || !uy || !uz || !w || !J.cell) return PXRB_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  if (J.prec == 0) k_load_particles<float><<<gs_blocks(J.np, 256), 256, 0, s>>>(J, x, y, z, ux, uy, uz, w);
  else k_load_particles<double><<<gs_blocks(J.np, 256), 256, 0, s>>>(J, x, y, z, ux, uy, uz, w);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_store_particles(const pxrb_tiled_job* job_host, double* x, double* y, double* z,
                               double* ux, double* uy, double* uz, double* gaminv, double* w,
                               void* stream) {
  if (!job_host) return PXRB_EINVAL;
  const Job& J = *job_host;
  if (J.np == 0) return PXRB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (J.prec == 0)
    k_store_particles<float><<<gs_blocks(J.np, 256), 256, 0, s>>>(J, x, y, z, ux, uy, uz, gaminv, w);
  else
    k_store_particles<double><<<gs_blocks(J.np, 256), 256, 0, s>>>(J, x, y, z, ux, uy, uz, gaminv, w);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

static int field_xfer(const pxrb_tiled_job* job_host, int32_t which, double* f, int64_t ng,
                      int dir, void* stream) {
  if (!job_host || !f || which < 0 || which > 8 || ng < 0) return PXRB_EINVAL;
  const Job& J = *job_host;
  cudaStream_t s = (cudaStream_t)stream;
  i64 total = (i64)(J.nx + 1 + 2 * ng) * (J.ny + 1 + 2 * ng) * (J.nz + 1 + 2 * ng);
  i64 t2 = (i64)(J.nx + 2 * J.g) * (J.ny + 2 * J.g) * (J.nz + 2 * J.g);
  if (t2 > total) total = t2;
  if (J.prec == 0) k_field_xfer<float><<<gs_blocks(total, 256), 256, 0, s>>>(J, which, f, (int)ng, dir);
  else k_field_xfer<double><<<gs_blocks(total, 256), 256, 0, s>>>(J, which, f, (int)ng, dir);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_tiled_field_import(const pxrb_tiled_job* job_host, int32_t which, const double* src,
                            int64_t nguard_src, void* stream) {
  return field_xfer(job_host, which, const_cast<double*>(src), nguard_src, 0, stream);
}

int pxrb_tiled_field_export(const pxrb_tiled_job* job_host, int32_t which, double* dst,
                            int64_t nguard_dst, void* stream) {
  return field_xfer(job_host, which, dst, nguard_dst, 1, stream);
}

int64_t pxrb_tiled_diag_scratch(const pxrb_tiled_job* job_host) {
  if (!job_host) return -1;
  return 8 * (int64_t)diag_blocks(*job_host);
}

int pxrb_tiled_diagnostics(const pxrb_tiled_job* job_host, double* rho, double* scratch,
                           int64_t scratch_len, double* out, void* stream) {
  if (!job_host || !scratch || !out) return PXRB_EINVAL;
  const Job& J = *job_host;
  const int nb = diag_blocks(J);
  if (scratch_len < 8 * (int64_t)nb) return PXRB_ESCRATCH;
  cudaStream_t s = (cudaStream_t)stream;
  if (rho && cudaMemsetAsync(rho, 0, sizeof(double) * (size_t)J.nx * J.ny * J.nz, s) != cudaSuccess)
    return PXRB_ELAUNCH;
  if (rho && J.np > 0) {
    const int pb = gs_blocks(J.np, 256);
#define PXRB_RHO(R_)                                                   \
    if (J.order == 1) k_rho_t<R_, 1><<<pb, 256, 0, s>>>(J, rho);       \
    else if (J.order == 2) k_rho_t<R_, 2><<<pb, 256, 0, s>>>(J, rho);  \
    else k_rho_t<R_, 3><<<pb, 256, 0, s>>>(J, rho);
    if (J.prec == 0) { PXRB_RHO(float) } else { PXRB_RHO(double) }
#undef PXRB_RHO
  }
  if (J.prec == 0) k_field_sums<float><<<nb, RED_TPB, 0, s>>>(J, rho, scratch);
  else k_field_sums<double><<<nb, RED_TPB, 0, s>>>(J, rho, scratch);
  k_diag_final<<<1, 32, 0, s>>>(J, scratch, nb, out);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

}  // extern "C"
