// Plain FP64 path: the drop-in kernels behind PICSAR's Forthon-exposed
// routines, on PICSAR's own guarded column-major FP64 arrays.  One thread per
// particle; deposition uses global FP64 atomics.  This is also the "plain
// FP64 GPU" baseline every mixed-precision / tiled speed-up is stated against.
#include "pxr_common.cuh"
#include "picsar_b200.h"

namespace {

constexpr int TPB = 256;

inline int nblocks(i64 n, int tpb = TPB) {
  i64 b = (n + tpb - 1) / tpb;
  return (int)(b < 1 ? 1 : (b > 2147483647 ? 2147483647 : b));
}

// ---------------------------------------------------------------------------
// Energy-conserving gather (accumulates) with the staggering of the fused
// kernels: E_c staggered along c, B_c staggered along the two other axes.
// Summation: for each z point, a = sum_y (sum_x s_x g) s_y; f += a s_z.
// ---------------------------------------------------------------------------
template <int NA, int NB, int NC>
__device__ __forceinline__ double gather_comp(const double* __restrict__ g, const GridG& G,
                                              int ia, const double* sa, int ib,
                                              const double* sb, int ic, const double* sc,
                                              double f) {
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    double a = 0.0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const double* row = g + G.idx(ia, ib + b, ic + c);
      double r = 0.0;
#pragma unroll
      for (int t = 0; t < NA; ++t) r = r + sa[t] * __ldg(row + t);
      a = a + r * sb[b];
    }
    f = f + a * sc[c];
  }
  return f;
}

template <int ORDER>
__device__ __forceinline__ void gather_eb(double x, double y, double z, const GridG& G,
                                          const double* exg, const double* eyg,
                                          const double* ezg, const double* bxg,
                                          const double* byg, const double* bzg, double& ex,
                                          double& ey, double& ez, double& bx, double& by,
                                          double& bz) {
  NodeShape<ORDER, double> nx, ny, nz;
  StagShape<ORDER, double> sx, sy, sz;
  nx.set(x); ny.set(y); nz.set(z);
  sx.set(x); sy.set(y); sz.set(z);
  constexpr int N = ORDER + 1, S = ORDER;
  ex = gather_comp<S, N, N>(exg, G, sx.i0, sx.s, ny.i0, ny.s, nz.i0, nz.s, ex);
  ey = gather_comp<N, S, N>(eyg, G, nx.i0, nx.s, sy.i0, sy.s, nz.i0, nz.s, ey);
  ez = gather_comp<N, N, S>(ezg, G, nx.i0, nx.s, ny.i0, ny.s, sz.i0, sz.s, ez);
  bx = gather_comp<N, S, S>(bxg, G, nx.i0, nx.s, sy.i0, sy.s, sz.i0, sz.s, bx);
  by = gather_comp<S, N, S>(byg, G, sx.i0, sx.s, ny.i0, ny.s, sz.i0, sz.s, by);
  bz = gather_comp<S, S, N>(bzg, G, sx.i0, sx.s, sy.i0, sy.s, nz.i0, nz.s, bz);
}

struct GPParams {
  i64 np;
  double *xp, *yp, *zp, *uxp, *uyp, *uzp, *gaminv;
  double *ex, *ey, *ez, *bx, *by, *bz;
  double xmin, ymin, zmin, dxi, dyi, dzi;
  const double *exg, *eyg, *ezg, *bxg, *byg, *bzg;
  GridG G;
  double q, m, dt, clight;
};

// field_gathering_plus_particle_pusher_{n}_{n}_{n}: gather (+=) into the
// particle field arrays, then Boris + set_gamma (pusher 0) or Vay (1), then
// pushxyz, all with the module time step dt.
template <int ORDER, int PUSHER>
__global__ void __launch_bounds__(TPB) k_gather_push(GPParams p) {
  const double cst_b = p.q * p.dt * 0.5 / p.m;
  const double cst_v = p.q * p.dt / p.m;
  const double clghtisq = 1.0 / (p.clight * p.clight);
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    double x = (p.xp[i] - p.xmin) * p.dxi;
    double y = (p.yp[i] - p.ymin) * p.dyi;
    double z = (p.zp[i] - p.zmin) * p.dzi;
    double ex = p.ex[i], ey = p.ey[i], ez = p.ez[i];
    double bx = p.bx[i], by = p.by[i], bz = p.bz[i];
    gather_eb<ORDER>(x, y, z, p.G, p.exg, p.eyg, p.ezg, p.bxg, p.byg, p.bzg, ex, ey, ez, bx,
                     by, bz);
    p.ex[i] = ex; p.ey[i] = ey; p.ez[i] = ez;
    p.bx[i] = bx; p.by[i] = by; p.bz[i] = bz;
    double ux = p.uxp[i], uy = p.uyp[i], uz = p.uzp[i], gi = p.gaminv[i];
    if (PUSHER == 1) {
      vay_push(ux, uy, uz, gi, ex, ey, ez, bx, by, bz, cst_v, 1.0 / p.clight, clghtisq);
    } else {
      boris_push(ux, uy, uz, gi, ex, ey, ez, bx, by, bz, cst_b, clghtisq);
      set_gamma(ux, uy, uz, gi, clghtisq);
    }
    p.uxp[i] = ux; p.uyp[i] = uy; p.uzp[i] = uz; p.gaminv[i] = gi;
    p.xp[i] = p.xp[i] + ux * gi * p.dt;
    p.yp[i] = p.yp[i] + uy * gi * p.dt;
    p.zp[i] = p.zp[i] + uz * gi * p.dt;
  }
}

// Separate gather (geteb3d_energy_conserving), both l_lower_order_in_v
// branches and the nodal switch; accumulates.  Generic over the order with
// run-time shapes (the scalar Fortran forms, field_gathering_o{1,2,3}_3d.F90).
struct Sh {
  int i0, n;
  double s[4];
};

__device__ __forceinline__ void sh_node(int order, double x, Sh& r) {
  if (order == 1) {
    int j = (int)floor(x); double xi = x - j;
    r.i0 = j; r.n = 2; r.s[0] = 1.0 - xi; r.s[1] = xi;
  } else if (order == 2) {
    int j = (int)round(x); double xi = x - j, xs = xi * xi;
    r.i0 = j - 1; r.n = 3;
    r.s[0] = 0.5 * (0.5 - xi) * (0.5 - xi); r.s[1] = 0.75 - xs; r.s[2] = 0.5 * (0.5 + xi) * (0.5 + xi);
  } else {
    int j = (int)floor(x); double xi = x - j, ox = 1.0 - xi, xs = xi * xi, oxs = ox * ox;
    r.i0 = j - 1; r.n = 4;
    r.s[0] = (1.0 / 6.0) * oxs * ox; r.s[1] = (2.0 / 3.0) - xs * (1.0 - xi * 0.5);
    r.s[2] = (2.0 / 3.0) - oxs * (1.0 - ox * 0.5); r.s[3] = (1.0 / 6.0) * xs * xi;
  }
}

__device__ __forceinline__ void sh_stag(int order, bool lower, double ss, double x, Sh& r) {
  if (order == 1) {
    if (lower) { r.i0 = (int)floor(x + 0.5 - ss); r.n = 1; r.s[0] = 1.0; }
    else {
      int j0 = (int)floor(x - ss); double xi = x - ss - j0;
      r.i0 = j0; r.n = 2; r.s[0] = 1.0 - xi; r.s[1] = xi;
    }
  } else if (order == 2) {
    if (lower) {
      int j0 = (int)floor(x - ss); double xi = x - ss - j0;
      r.i0 = j0; r.n = 2; r.s[0] = 1.0 - xi; r.s[1] = xi;
    } else {
      int j0 = (int)floor(x + 0.5 - ss); double xi = x - ss - j0, xs = xi * xi;
      r.i0 = j0 - 1; r.n = 3;
      r.s[0] = 0.5 * (0.5 - xi) * (0.5 - xi); r.s[1] = 0.75 - xs; r.s[2] = 0.5 * (0.5 + xi) * (0.5 + xi);
    }
  } else {
    if (lower) {
      int j0 = (int)floor(x + 0.5 - ss); double xi = x - ss - j0, xs = xi * xi;
      r.i0 = j0 - 1; r.n = 3;
      r.s[0] = 0.5 * (0.5 - xi) * (0.5 - xi); r.s[1] = 0.75 - xs; r.s[2] = 0.5 * (0.5 + xi) * (0.5 + xi);
    } else {
      int j0 = (int)floor(x - ss); double xi = x - ss - j0, ox = 1.0 - xi, xs = xi * xi, oxs = ox * ox;
      r.i0 = j0 - 1; r.n = 4;
      r.s[0] = (1.0 / 6.0) * oxs * ox; r.s[1] = (2.0 / 3.0) - xs * (1.0 - xi * 0.5);
      r.s[2] = (2.0 / 3.0) - oxs * (1.0 - ox * 0.5); r.s[3] = (1.0 / 6.0) * xs * xi;
    }
  }
}

__device__ __forceinline__ double gsum(const double* g, const GridG& G, const Sh& a,
                                       const Sh& b, const Sh& c, double f) {
  for (int ll = 0; ll < c.n; ++ll)
    for (int kk = 0; kk < b.n; ++kk)
      for (int jj = 0; jj < a.n; ++jj)
        f = f + a.s[jj] * b.s[kk] * c.s[ll] * __ldg(g + G.idx(a.i0 + jj, b.i0 + kk, c.i0 + ll));
  return f;
}

struct GEBParams {
  i64 np;
  const double *xp, *yp, *zp;
  double *ex, *ey, *ez, *bx, *by, *bz;
  double xmin, ymin, zmin, dxi, dyi, dzi;
  const double *exg, *eyg, *ezg, *bxg, *byg, *bzg;
  GridG G;
  int order, lower;
  double ss;
};

__global__ void __launch_bounds__(TPB) k_geteb(GEBParams p) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    double x = (p.xp[i] - p.xmin) * p.dxi, y = (p.yp[i] - p.ymin) * p.dyi,
           z = (p.zp[i] - p.zmin) * p.dzi;
    Sh nx, ny, nz, sx, sy, sz;
    sh_node(p.order, x, nx); sh_node(p.order, y, ny); sh_node(p.order, z, nz);
    sh_stag(p.order, p.lower, p.ss, x, sx);
    sh_stag(p.order, p.lower, p.ss, y, sy);
    sh_stag(p.order, p.lower, p.ss, z, sz);
    p.ex[i] = gsum(p.exg, p.G, sx, ny, nz, p.ex[i]);
    p.ey[i] = gsum(p.eyg, p.G, nx, sy, nz, p.ey[i]);
    p.ez[i] = gsum(p.ezg, p.G, nx, ny, sz, p.ez[i]);
    p.bx[i] = gsum(p.bxg, p.G, nx, sy, sz, p.bx[i]);
    p.by[i] = gsum(p.byg, p.G, sx, ny, sz, p.by[i]);
    p.bz[i] = gsum(p.bzg, p.G, sx, sy, nz, p.bz[i]);
  }
}

// ---------------------------------------------------------------------------
// Stand-alone pushers.
// ---------------------------------------------------------------------------
struct PushParams {
  i64 np;
  double *ux, *uy, *uz, *gi;
  const double *ex, *ey, *ez, *bx, *by, *bz;
  double *x, *y, *z;
  double q, m, dt, clight;
  int which;
};

__global__ void k_boris(PushParams p) {
  const double cst = p.q * p.dt * 0.5 / p.m, c2i = 1.0 / (p.clight * p.clight);
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    double ux = p.ux[i], uy = p.uy[i], uz = p.uz[i], gi = p.gi[i];
    boris_push(ux, uy, uz, gi, p.ex[i], p.ey[i], p.ez[i], p.bx[i], p.by[i], p.bz[i], cst, c2i);
    p.ux[i] = ux; p.uy[i] = uy; p.uz[i] = uz; p.gi[i] = gi;
  }
}

__global__ void k_vay(PushParams p) {
  const double invc = 1.0 / p.clight, invc2 = 1.0 / (p.clight * p.clight);
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    double ux = p.ux[i], uy = p.uy[i], uz = p.uz[i], gi = p.gi[i];
    double ex = p.ex[i], ey = p.ey[i], ez = p.ez[i], bx = p.bx[i], by = p.by[i], bz = p.bz[i];
    if (p.which == 0) {
      vay_push(ux, uy, uz, gi, ex, ey, ez, bx, by, bz, p.q * p.dt / p.m, invc, invc2);
    } else if (p.which == 1) {
      const double cst = 0.5 * p.q * p.dt / p.m;
      double vx = ux * gi, vy = uy * gi, vz = uz * gi;
      ux = ux + cst * (ex + vy * bz - vz * by);
      uy = uy + cst * (ey + vz * bx - vx * bz);
      uz = uz + cst * (ez + vx * by - vy * bx);
      gi = 1.0 / sqrt(1.0 + (ux * ux + uy * uy + uz * uz) * invc2);
    } else {
      const double cst = 0.5 * p.q * p.dt / p.m, bconst = cst;
      double uxpr = ux + cst * ex, uypr = uy + cst * ey, uzpr = uz + cst * ez;
      double gprsq = (1.0 + (uxpr * uxpr + uypr * uypr + uzpr * uzpr) * invc2);
      double taux = bconst * bx, tauy = bconst * by, tauz = bconst * bz;
      double tausq = taux * taux + tauy * tauy + tauz * tauz;
      double ust = (uxpr * taux + uypr * tauy + uzpr * tauz) * invc;
      double sigma = gprsq - tausq;
      double gisq = 2.0 / (sigma + sqrt(sigma * sigma + 4.0 * (tausq + ust * ust)));
      gi = sqrt(gisq);
      double bg = bconst * gi, tx = bg * bx, ty = bg * by, tz = bg * bz;
      double s = 1.0 / (1.0 + tausq * gisq);
      double tu = tx * uxpr + ty * uypr + tz * uzpr;
      ux = s * (uxpr + tx * tu + uypr * tz - uzpr * ty);
      uy = s * (uypr + ty * tu + uzpr * tx - uxpr * tz);
      uz = s * (uzpr + tz * tu + uxpr * ty - uypr * tx);
    }
    p.ux[i] = ux; p.uy[i] = uy; p.uz[i] = uz; p.gi[i] = gi;
  }
}

__global__ void k_set_gamma(PushParams p) {
  const double c2i = 1.0 / (p.clight * p.clight);
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    double gi;
    set_gamma(p.ux[i], p.uy[i], p.uz[i], gi, c2i);
    p.gi[i] = gi;
  }
}

__global__ void k_pushxyz(PushParams p) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    double gi = p.gi[i];
    p.x[i] = p.x[i] + p.ux[i] * gi * p.dt;
    p.y[i] = p.y[i] + p.uy[i] * gi * p.dt;
    p.z[i] = p.z[i] + p.uz[i] * gi * p.dt;
  }
}

// ---------------------------------------------------------------------------
// Esirkepov deposition with global FP64 atomics.  The old position is
// reconstructed as x - dt/dx*ux*gaminv (esirkepov_3d.F90:161-163); for the
// generic "_n" entry (reconstruct = 1) the new position is recomputed as
// xold + dt/dx*v as that routine does (:3566-3577).
// Currents are prefix sums of W along x (Jx), y (Jy), z (Jz) over the box.
// ---------------------------------------------------------------------------
struct DepParams {
  i64 np;
  const double *xp, *yp, *zp, *uxp, *uyp, *uzp, *gaminv, *w;
  double *jx, *jy, *jz;
  GridG G;
  double q, xmin, ymin, zmin, dxi, dyi, dzi, dtsdx, dtsdy, dtsdz;
  double invdtdx, invdtdy, invdtdz;
  int reconstruct;
  int* err;
};

template <int ORDER>
__device__ __forceinline__ void esir_axis(double x, double xold, EsirAxis<ORDER, double>& A,
                                          bool& ok) {
  int n0 = EsirAxis<ORDER, double>::node(x);
  int n1 = EsirAxis<ORDER, double>::node(xold);
  ok = A.set(n0, x - n0, n1, xold - n1) && ok;
}

template <int ORDER>
__global__ void __launch_bounds__(TPB) k_esirkepov(DepParams p) {
  constexpr int M = ORDER + 2;
  const double onethird = 1.0 / 3.0;
  for (i64 ip = blockIdx.x * (i64)blockDim.x + threadIdx.x; ip < p.np;
       ip += (i64)gridDim.x * blockDim.x) {
    double x = (p.xp[ip] - p.xmin) * p.dxi, y = (p.yp[ip] - p.ymin) * p.dyi,
           z = (p.zp[ip] - p.zmin) * p.dzi;
    double gi = p.gaminv[ip];
    double vx = p.uxp[ip] * gi, vy = p.uyp[ip] * gi, vz = p.uzp[ip] * gi;
    double xold = x - p.dtsdx * vx, yold = y - p.dtsdy * vy, zold = z - p.dtsdz * vz;
    if (p.reconstruct) {
      x = xold + p.dtsdx * vx; y = yold + p.dtsdy * vy; z = zold + p.dtsdz * vz;
    }
    double wq = p.q * p.w[ip];
    double wqx = wq * p.invdtdx, wqy = wq * p.invdtdy, wqz = wq * p.invdtdz;
    EsirAxis<ORDER, double> X, Y, Z;
    bool ok = true;
    esir_axis<ORDER>(x, xold, X, ok);
    esir_axis<ORDER>(y, yold, Y, ok);
    esir_axis<ORDER>(z, zold, Z, ok);
    if (!ok) { atomicExch(p.err, 1); continue; }
    // Jx: sweep x for every (j, k)
#pragma unroll
    for (int k = 0; k < M; ++k) {
      if (k >= Z.n) continue;
      double dsz = Z.s1[k] - Z.s0[k];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        if (j >= Y.n) continue;
        double dsy = Y.s1[j] - Y.s0[j];
        double fyz = (Y.s0[j] + 0.5 * dsy) * Z.s0[k] + (0.5 * Y.s0[j] + onethird * dsy) * dsz;
        double acc = 0.0;
        double* row = p.jx + p.G.idx(X.i0, Y.i0 + j, Z.i0 + k);
#pragma unroll
        for (int i = 0; i < M - 1; ++i) {
          if (i >= X.n - 1) continue;
          acc = acc + wqx * (X.s1[i] - X.s0[i]) * fyz;
          atomicAdd(row + i, acc);
        }
      }
    }
    // Jy: sweep y for every (i, k)
#pragma unroll
    for (int k = 0; k < M; ++k) {
      if (k >= Z.n) continue;
      double dsz = Z.s1[k] - Z.s0[k];
#pragma unroll
      for (int i = 0; i < M; ++i) {
        if (i >= X.n) continue;
        double dsx = X.s1[i] - X.s0[i];
        double fzx = (Z.s0[k] + 0.5 * dsz) * X.s0[i] + (0.5 * Z.s0[k] + onethird * dsz) * dsx;
        double acc = 0.0;
        double* col = p.jy + p.G.idx(X.i0 + i, Y.i0, Z.i0 + k);
#pragma unroll
        for (int j = 0; j < M - 1; ++j) {
          if (j >= Y.n - 1) continue;
          acc = acc + wqy * (Y.s1[j] - Y.s0[j]) * fzx;
          atomicAdd(col + j * p.G.sx, acc);
        }
      }
    }
    // Jz: sweep z for every (i, j)
#pragma unroll
    for (int j = 0; j < M; ++j) {
      if (j >= Y.n) continue;
      double dsy = Y.s1[j] - Y.s0[j];
#pragma unroll
      for (int i = 0; i < M; ++i) {
        if (i >= X.n) continue;
        double dsx = X.s1[i] - X.s0[i];
        double fxy = (X.s0[i] + 0.5 * dsx) * Y.s0[j] + (0.5 * X.s0[i] + onethird * dsx) * dsy;
        double acc = 0.0;
        double* col = p.jz + p.G.idx(X.i0 + i, Y.i0 + j, Z.i0);
#pragma unroll
        for (int k = 0; k < M - 1; ++k) {
          if (k >= Z.n - 1) continue;
          acc = acc + wqz * (Z.s1[k] - Z.s0[k]) * fxy;
          atomicAdd(col + k * p.G.sy, acc);
        }
      }
    }
  }
}

// Node-centred charge deposition (charge_deposition_3d.F90:77-400).
struct RhoParams {
  i64 np;
  const double *xp, *yp, *zp, *w;
  double* rho;
  GridG G;
  double q, xmin, ymin, zmin, dxi, dyi, dzi, invvol;
};

template <int ORDER>
__global__ void __launch_bounds__(TPB) k_rho(RhoParams p) {
  for (i64 ip = blockIdx.x * (i64)blockDim.x + threadIdx.x; ip < p.np;
       ip += (i64)gridDim.x * blockDim.x) {
    double x = (p.xp[ip] - p.xmin) * p.dxi, y = (p.yp[ip] - p.ymin) * p.dyi,
           z = (p.zp[ip] - p.zmin) * p.dzi;
    double wq = p.q * p.w[ip] * p.invvol;
    NodeShape<ORDER, double> sx, sy, sz;
    sx.set(x); sy.set(y); sz.set(z);
#pragma unroll
    for (int c = 0; c < ORDER + 1; ++c)
#pragma unroll
      for (int b = 0; b < ORDER + 1; ++b)
#pragma unroll
        for (int a = 0; a < ORDER + 1; ++a)
          atomicAdd(p.rho + p.G.idx(sx.i0 + a, sy.i0 + b, sz.i0 + c),
                    sx.s[a] * sy.s[b] * sz.s[c] * wq);
  }
}

// ---------------------------------------------------------------------------
// Yee (yee.F90:637-740, :1258-1347).  Thread (j,k,l) over the union of the
// three component ranges; each component predicated on its own range.
// ---------------------------------------------------------------------------
struct YeeParams {
  double *ex, *ey, *ez, *bx, *by, *bz;
  const double *jx, *jy, *jz;
  GridG gex, gey, gez, gbx, gby, gbz, gjx, gjy, gjz;  // per-array bounds
  int lo[3][3], hi[3][3];   // per-component loop ranges
  int ulo[3], uhi[3];       // union
  double mudt, dtsdx, dtsdy, dtsdz;
};

__device__ __forceinline__ bool inr(const int* lo, const int* hi, int j, int k, int l) {
  return j >= lo[0] && j <= hi[0] && k >= lo[1] && k <= hi[1] && l >= lo[2] && l <= hi[2];
}

__global__ void k_yee_e(YeeParams p) {
  int j = p.ulo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  int k = p.ulo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  int l = p.ulo[2] + blockIdx.z;
  if (j > p.uhi[0] || k > p.uhi[1] || l > p.uhi[2]) return;
  if (inr(p.lo[0], p.hi[0], j, k, l)) {
    double* e = p.ex + p.gex.idx(j, k, l);
    *e = *e + p.dtsdy * (p.bz[p.gbz.idx(j, k, l)] - p.bz[p.gbz.idx(j, k - 1, l)]) -
         p.dtsdz * (p.by[p.gby.idx(j, k, l)] - p.by[p.gby.idx(j, k, l - 1)]) -
         p.mudt * p.jx[p.gjx.idx(j, k, l)];
  }
  if (inr(p.lo[1], p.hi[1], j, k, l)) {
    double* e = p.ey + p.gey.idx(j, k, l);
    *e = *e - p.dtsdx * (p.bz[p.gbz.idx(j, k, l)] - p.bz[p.gbz.idx(j - 1, k, l)]) +
         p.dtsdz * (p.bx[p.gbx.idx(j, k, l)] - p.bx[p.gbx.idx(j, k, l - 1)]) -
         p.mudt * p.jy[p.gjy.idx(j, k, l)];
  }
  if (inr(p.lo[2], p.hi[2], j, k, l)) {
    double* e = p.ez + p.gez.idx(j, k, l);
    *e = *e + p.dtsdx * (p.by[p.gby.idx(j, k, l)] - p.by[p.gby.idx(j - 1, k, l)]) -
         p.dtsdy * (p.bx[p.gbx.idx(j, k, l)] - p.bx[p.gbx.idx(j, k - 1, l)]) -
         p.mudt * p.jz[p.gjz.idx(j, k, l)];
  }
}

__global__ void k_yee_b(YeeParams p) {
  int j = p.ulo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  int k = p.ulo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  int l = p.ulo[2] + blockIdx.z;
  if (j > p.uhi[0] || k > p.uhi[1] || l > p.uhi[2]) return;
  if (inr(p.lo[0], p.hi[0], j, k, l)) {
    double* b = p.bx + p.gbx.idx(j, k, l);
    *b = *b - p.dtsdy * (p.ez[p.gez.idx(j, k + 1, l)] - p.ez[p.gez.idx(j, k, l)]) +
         p.dtsdz * (p.ey[p.gey.idx(j, k, l + 1)] - p.ey[p.gey.idx(j, k, l)]);
  }
  if (inr(p.lo[1], p.hi[1], j, k, l)) {
    double* b = p.by + p.gby.idx(j, k, l);
    *b = *b + p.dtsdx * (p.ez[p.gez.idx(j + 1, k, l)] - p.ez[p.gez.idx(j, k, l)]) -
         p.dtsdz * (p.ex[p.gex.idx(j, k, l + 1)] - p.ex[p.gex.idx(j, k, l)]);
  }
  if (inr(p.lo[2], p.hi[2], j, k, l)) {
    double* b = p.bz + p.gbz.idx(j, k, l);
    *b = *b - p.dtsdx * (p.ey[p.gey.idx(j + 1, k, l)] - p.ey[p.gey.idx(j, k, l)]) +
         p.dtsdy * (p.ex[p.gex.idx(j, k + 1, l)] - p.ex[p.gex.idx(j, k, l)]);
  }
}

// ---------------------------------------------------------------------------
// Periodic single-domain guard exchanges, one kernel per axis for up to three
// arrays; each thread owns one line along the axis and performs the slab
// operations of field_bc / summation_bcs in their sequential order
// (field_boundaries.F90:107-269 and :403-503).  Requires n > g per axis so
// source and destination slabs never overlap within the line.
// ---------------------------------------------------------------------------
struct BcParams {
  double* a[3];
  int na;
  GridG G;
  int axis;
  int mode;  // 0: field_bc (copy), 1: summation (fold-add)
};

__global__ void k_bc_axis(BcParams p) {
  const GridG& G = p.G;
  i64 ext[3] = {G.nx + 1 + 2 * G.gx, G.ny + 1 + 2 * G.gy, G.nz + 1 + 2 * G.gz};
  i64 str[3] = {1, G.sx, G.sy};
  i64 n[3] = {G.nx, G.ny, G.nz}, g[3] = {G.gx, G.gy, G.gz};
  int ax = p.axis, a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
  // lines are indexed by the other two axes (lower one fastest)
  int lo_ax = a1 < a2 ? a1 : a2, hi_ax = a1 < a2 ? a2 : a1;
  i64 nlines = ext[lo_ax] * ext[hi_ax];
  i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
  if (t >= nlines) return;
  i64 c_lo = t % ext[lo_ax], c_hi = t / ext[lo_ax];
  i64 base = c_lo * str[lo_ax] + c_hi * str[hi_ax];  // offset of storage index 0 on axis
  i64 s = str[ax], N = n[ax], Gd = g[ax];
  // storage index of node i is i + Gd
  for (int q = 0; q < p.na; ++q) {
    double* L = p.a[q] + base;
    if (p.mode == 0) {
      // A[n+i] = A[i], i = 0..g ; then A[-g+i] = A[n-g+i], i = 0..g
      for (i64 i = 0; i <= Gd; ++i) L[(N + i + Gd) * s] = L[(i + Gd) * s];
      for (i64 i = 0; i <= Gd; ++i) L[(-Gd + i + Gd) * s] = L[(N - Gd + i + Gd) * s];
    } else {
      // A[i] += A[n+i], i = 0..g ; then A[n-g+i] += A[-g+i], i = 0..g
      for (i64 i = 0; i <= Gd; ++i) L[(i + Gd) * s] = L[(i + Gd) * s] + L[(N + i + Gd) * s];
      for (i64 i = 0; i <= Gd; ++i)
        L[(N - Gd + i + Gd) * s] = L[(N - Gd + i + Gd) * s] + L[(i) * s];
    }
  }
}

// Periodic particle wrap (particle_boundaries.F90:1109-1300, pbound = 0).
struct WrapParams {
  i64 np;
  double *x, *y, *z;
  double lo[3], hi[3];
};

__global__ void k_wrap(WrapParams p) {
  double len[3] = {p.hi[0] - p.lo[0], p.hi[1] - p.lo[1], p.hi[2] - p.lo[2]};
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    double* c[3] = {p.x + i, p.y + i, p.z + i};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double v = *c[a];
      if (v < p.lo[a]) *c[a] = v + len[a];
      else if (v >= p.hi[a]) *c[a] = v - len[a];
    }
  }
}

inline int grid_stride_blocks(i64 n) {
  // enough CTAs to fill 148 SMs several times over, capped by the work
  i64 b = (n + TPB - 1) / TPB;
  const i64 cap = 148 * 16;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

bool bad_ptr(const void* p) { return p == nullptr; }

// ---------------------------------------------------------------------------
// 2D (x-z) path on PICSAR's 2-D arrays (-g:n+g) in x and z, Fortran order:
// the separate energy-conserving gather (field_gathering_o{1,2,3}_2d.F90),
// Esirkepov deposition (esirkepov_2d.F90:452-1082) with global FP64 atomics,
// the order-2 Yee update (yee.F90:216-310, :912-994) and pxr_pushxz.
// ---------------------------------------------------------------------------
struct G2 {
  i64 gx, gz, sx;
  __device__ __forceinline__ i64 idx(i64 i, i64 k) const { return (i + gx) + sx * (k + gz); }
};

__device__ __forceinline__ double gsum2(const double* g, const G2& G, const Sh& a, const Sh& c,
                                        double f) {
  for (int ll = 0; ll < c.n; ++ll)
    for (int jj = 0; jj < a.n; ++jj)
      f = f + a.s[jj] * c.s[ll] * __ldg(g + G.idx(a.i0 + jj, c.i0 + ll));
  return f;
}

struct GEB2Params {
  i64 np;
  const double *xp, *zp;
  double *ex, *ey, *ez, *bx, *by, *bz;
  double xmin, zmin, dxi, dzi;
  const double *exg, *eyg, *ezg, *bxg, *byg, *bzg;
  G2 G;
  int order, lower;
  double ss;
};

__global__ void __launch_bounds__(TPB) k_geteb2d(GEB2Params p) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < p.np;
       i += (i64)gridDim.x * blockDim.x) {
    const double x = (p.xp[i] - p.xmin) * p.dxi, z = (p.zp[i] - p.zmin) * p.dzi;
    Sh nx, nz, sx, sz;
    sh_node(p.order, x, nx); sh_node(p.order, z, nz);
    sh_stag(p.order, p.lower, p.ss, x, sx); sh_stag(p.order, p.lower, p.ss, z, sz);
    p.ex[i] = gsum2(p.exg, p.G, sx, nz, p.ex[i]);
    p.ey[i] = gsum2(p.eyg, p.G, nx, nz, p.ey[i]);
    p.ez[i] = gsum2(p.ezg, p.G, nx, sz, p.ez[i]);
    p.bx[i] = gsum2(p.bxg, p.G, nx, sz, p.bx[i]);
    p.by[i] = gsum2(p.byg, p.G, sx, sz, p.by[i]);
    p.bz[i] = gsum2(p.bzg, p.G, sx, nz, p.bz[i]);
  }
}

struct Dep2Params {
  i64 np;
  double *jx, *jy, *jz;
  const double *xp, *zp, *uxp, *uyp, *uzp, *gaminv, *w;
  double q, xmin, zmin, dt, dx, dz;
  G2 G;
};

// The reference's 2-D shapes: order 3 with its default-real (single
// precision) constants 1/6 and 2/3; array index off = shift of the shape.
template <int ORDER>
__device__ __forceinline__ void shape2d(double xint, double* s, int off) {
  if (ORDER == 1) {
    s[0 + off] = 1.0 - xint; s[1 + off] = xint;
  } else if (ORDER == 2) {
    const double xs = xint * xint;
    s[-1 + off] = 0.5 * (0.5 - xint) * (0.5 - xint);
    s[0 + off] = 0.75 - xs;
    s[1 + off] = 0.5 * (0.5 + xint) * (0.5 + xint);
  } else {
    const double onesixth = (double)(1.0f / 6.0f), twothird = (double)(2.0f / 3.0f);
    const double ox = 1.0 - xint, xs = xint * xint, oxs = ox * ox;
    s[-1 + off] = onesixth * oxs * ox;
    s[0 + off] = twothird - xs * (1.0 - xint * 0.5);
    s[1 + off] = twothird - oxs * (1.0 - ox * 0.5);
    s[2 + off] = onesixth * xs * xint;
  }
}

template <int ORDER>
__global__ void __launch_bounds__(TPB) k_esirkepov2d(Dep2Params p) {
  constexpr int a = ORDER == 1 ? 0 : 1, b = ORDER == 3 ? 2 : 1;
  const double onethird = (double)(1.0f / 3.0f);
  const double dxi = 1.0 / p.dx, dzi = 1.0 / p.dz;
  const double dtsdx0 = p.dt * dxi, dtsdz0 = p.dt * dzi;
  const double invvol = 1.0 / (p.dx * p.dz), invdtdx = 1.0 / (p.dt * p.dz),
               invdtdz = 1.0 / (p.dt * p.dx);
  for (i64 ip = blockIdx.x * (i64)blockDim.x + threadIdx.x; ip < p.np;
       ip += (i64)gridDim.x * blockDim.x) {
    // (-2:3) arrays at offset +2
    double sx_[6] = {0, 0, 0, 0, 0, 0}, sz_[6] = {0, 0, 0, 0, 0, 0};
    double sx0_[6] = {0, 0, 0, 0, 0, 0}, sz0_[6] = {0, 0, 0, 0, 0, 0};
    double sdzk_[6] = {0, 0, 0, 0, 0, 0}, sdzkm1_[6] = {0, 0, 0, 0, 0, 0};
    double *sx = sx_ + 2, *sz = sz_ + 2, *sx0 = sx0_ + 2, *sz0 = sz0_ + 2;
    double *sdzk = sdzk_ + 2, *sdzkm1 = sdzkm1_ + 2;
    const double x = (p.xp[ip] - p.xmin) * dxi, z = (p.zp[ip] - p.zmin) * dzi;
    const double gi = p.gaminv[ip];
    const double vx = p.uxp[ip] * gi, vy = p.uyp[ip] * gi, vz = p.uzp[ip] * gi;
    const double xold = x - dtsdx0 * vx, zold = z - dtsdz0 * vz;
    const double wq = p.q * p.w[ip], wqx = wq * invdtdx, wqz = wq * invdtdz;
    const i64 iixp0 = ORDER == 2 ? (i64)round(x) : (i64)floor(x);
    const i64 ikxp0 = ORDER == 2 ? (i64)round(z) : (i64)floor(z);
    shape2d<ORDER>(x - iixp0, sx0, 0);
    shape2d<ORDER>(z - ikxp0, sz0, 0);
    const i64 iixp = ORDER == 2 ? (i64)round(xold) : (i64)floor(xold);
    const i64 ikxp = ORDER == 2 ? (i64)round(zold) : (i64)floor(zold);
    int dix = (int)(iixp - iixp0), diz = (int)(ikxp - ikxp0);
    // a move of more than one cell per step (beyond the CFL limit) would
    // leave the shape arrays: clamp, as no valid input reaches it
    dix = dix < -1 ? -1 : (dix > 1 ? 1 : dix);
    diz = diz < -1 ? -1 : (diz > 1 ? 1 : diz);
    shape2d<ORDER>(xold - iixp, sx, dix);
    shape2d<ORDER>(zold - ikxp, sz, diz);
    const int ixmin = min(0, dix) - a, ixmax = max(0, dix) + b;
    const int izmin = min(0, diz) - a, izmax = max(0, diz) + b;
    double sdxi = 0.0, sdxim1 = 0.0;
    for (int k = izmin; k <= izmax; ++k) {
      const double dsz = sz[k] - sz0[k];
      for (int i = ixmin; i <= ixmax; ++i) {
        const double dsx = sx[i] - sx0[i];
        const i64 c = p.G.idx(iixp0 + i, ikxp0 + k);
        if (i < ixmax) {
          sdxi = wqx * dsx * (sz0[k] + 0.5 * dsz);
          if (i > ixmin) sdxi = sdxi + sdxim1;
          atomicAdd(p.jx + c, sdxi);
        }
        atomicAdd(p.jy + c, wq * vy * invvol *
                                ((sz0[k] + 0.5 * dsz) * sx0[i] + (0.5 * sz0[k] + onethird * dsz) * dsx));
        if (k < izmax) {
          sdzk[i] = wqz * dsz * (sx0[i] + 0.5 * dsx);
          if (k > izmin) sdzk[i] = sdzk[i] + sdzkm1[i];
          atomicAdd(p.jz + c, sdzk[i]);
        }
        sdxim1 = sdxi;
      }
      for (int t = 0; t < 6; ++t) sdzkm1_[t] = sdzk_[t];
    }
  }
}

struct Yee2Params {
  double *ex, *ey, *ez, *bx, *by, *bz;
  const double *jx, *jy, *jz;
  G2 gex, gey, gez, gbx, gby, gbz, gjx, gjy, gjz;
  int lo[3][2], hi[3][2];
  int ulo[2], uhi[2];
  double mudt, dtsdx, dtsdz;
};

__device__ __forceinline__ bool inr2(const int* lo, const int* hi, int j, int k) {
  return j >= lo[0] && j <= hi[0] && k >= lo[1] && k <= hi[1];
}

__global__ void k_yee2d_e(Yee2Params p) {
  const int j = p.ulo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  const int k = p.ulo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  if (j > p.uhi[0] || k > p.uhi[1]) return;
  if (inr2(p.lo[0], p.hi[0], j, k)) {
    double* e = p.ex + p.gex.idx(j, k);
    *e = *e - p.dtsdz * (p.by[p.gby.idx(j, k)] - p.by[p.gby.idx(j, k - 1)]) -
         p.mudt * p.jx[p.gjx.idx(j, k)];
  }
  if (inr2(p.lo[1], p.hi[1], j, k)) {
    double* e = p.ey + p.gey.idx(j, k);
    *e = *e - p.dtsdx * (p.bz[p.gbz.idx(j, k)] - p.bz[p.gbz.idx(j - 1, k)]) +
         p.dtsdz * (p.bx[p.gbx.idx(j, k)] - p.bx[p.gbx.idx(j, k - 1)]) -
         p.mudt * p.jy[p.gjy.idx(j, k)];
  }
  if (inr2(p.lo[2], p.hi[2], j, k)) {
    double* e = p.ez + p.gez.idx(j, k);
    *e = *e + p.dtsdx * (p.by[p.gby.idx(j, k)] - p.by[p.gby.idx(j - 1, k)]) -
         p.mudt * p.jz[p.gjz.idx(j, k)];
  }
}

__global__ void k_yee2d_b(Yee2Params p) {
  const int j = p.ulo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  const int k = p.ulo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  if (j > p.uhi[0] || k > p.uhi[1]) return;
  if (inr2(p.lo[0], p.hi[0], j, k)) {
    double* b = p.bx + p.gbx.idx(j, k);
    *b = *b + p.dtsdz * (p.ey[p.gey.idx(j, k + 1)] - p.ey[p.gey.idx(j, k)]);
  }
  if (inr2(p.lo[1], p.hi[1], j, k)) {
    double* b = p.by + p.gby.idx(j, k);
    *b = *b + p.dtsdx * (p.ez[p.gez.idx(j + 1, k)] - p.ez[p.gez.idx(j, k)]) -
         p.dtsdz * (p.ex[p.gex.idx(j, k + 1)] - p.ex[p.gex.idx(j, k)]);
  }
  if (inr2(p.lo[2], p.hi[2], j, k)) {
    double* b = p.bz + p.gbz.idx(j, k);
    *b = *b - p.dtsdx * (p.ey[p.gey.idx(j + 1, k)] - p.ey[p.gey.idx(j, k)]);
  }
}

__global__ void k_pushxz(i64 np, double* xp, double* zp, const double* uxp, const double* uzp,
                         const double* gaminv, double dt) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < np;
       i += (i64)gridDim.x * blockDim.x) {
    xp[i] = xp[i] + uxp[i] * gaminv[i] * dt;
    zp[i] = zp[i] + uzp[i] * gaminv[i] * dt;
  }
}

inline G2 g2_lohi(const int64_t* lo, const int64_t* hi) {
  G2 g;
  g.gx = -lo[0]; g.gz = -lo[1];
  g.sx = hi[0] - lo[0] + 1;
  return g;
}

}  // namespace

// ===========================================================================
// extern "C" entry points
// ===========================================================================
extern "C" {

int pxrb_field_gathering_plus_particle_pusher(
    int64_t order, int64_t np, double* xp, double* yp, double* zp, double* uxp, double* uyp,
    double* uzp, double* gaminv, double* ex, double* ey, double* ez, double* bx, double* by,
    double* bz, double xmin, double ymin, double zmin, double dx, double dy, double dz,
    double dtt, int64_t nx, int64_t ny, int64_t nz, int64_t nxguard, int64_t nyguard,
    int64_t nzguard, const double* exg, const double* eyg, const double* ezg,
    const double* bxg, const double* byg, const double* bzg, double q, double m,
    int64_t lvect, int64_t l_lower_order_in_v, double dt, int64_t particle_pusher,
    double clight, void* stream) {
  (void)dtt; (void)lvect;
  if (np < 0 || nx < 0 || ny < 0 || nz < 0) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  if (order < 1 || order > 3 || !l_lower_order_in_v) return PXRB_EUNSUPPORTED;
  const void* ptrs[] = {xp, yp, zp, uxp, uyp, uzp, gaminv, ex, ey, ez, bx, by, bz,
                        exg, eyg, ezg, bxg, byg, bzg};
  for (const void* p : ptrs) if (bad_ptr(p)) return PXRB_EINVAL;
  GPParams p;
  p.np = np; p.xp = xp; p.yp = yp; p.zp = zp; p.uxp = uxp; p.uyp = uyp; p.uzp = uzp;
  p.gaminv = gaminv; p.ex = ex; p.ey = ey; p.ez = ez; p.bx = bx; p.by = by; p.bz = bz;
  p.xmin = xmin; p.ymin = ymin; p.zmin = zmin;
  p.dxi = 1.0 / dx; p.dyi = 1.0 / dy; p.dzi = 1.0 / dz;
  p.exg = exg; p.eyg = eyg; p.ezg = ezg; p.bxg = bxg; p.byg = byg; p.bzg = bzg;
  p.G = make_grid(nx, ny, nz, nxguard, nyguard, nzguard);
  p.q = q; p.m = m; p.dt = dt; p.clight = clight;
  cudaStream_t s = (cudaStream_t)stream;
  int nb = nblocks(np);
  int vay = particle_pusher == 1;
#define LAUNCH_GP(O)                                                                   \
  if (vay) k_gather_push<O, 1><<<nb, TPB, 0, s>>>(p);                                  \
  else k_gather_push<O, 0><<<nb, TPB, 0, s>>>(p);
  if (order == 1) { LAUNCH_GP(1) }
  else if (order == 2) { LAUNCH_GP(2) }
  else { LAUNCH_GP(3) }
#undef LAUNCH_GP
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

#define PXRB_FGP_N(O)                                                                   \
  int pxrb_field_gathering_plus_particle_pusher_##O##_##O##_##O(                          \
      int64_t np, double* xp, double* yp, double* zp, double* uxp, double* uyp,           \
      double* uzp, double* gaminv, double* ex, double* ey, double* ez, double* bx,        \
      double* by, double* bz, double xmin, double ymin, double zmin, double dx, double dy, \
      double dz, double dtt, int64_t nx, int64_t ny, int64_t nz, int64_t nxguard,         \
      int64_t nyguard, int64_t nzguard, const double* exg, const double* eyg,             \
      const double* ezg, const double* bxg, const double* byg, const double* bzg,         \
      double q, double m, int64_t lvect, int64_t l_lower_order_in_v, double dt,           \
      int64_t particle_pusher, double clight, void* stream) {                             \
    return pxrb_field_gathering_plus_particle_pusher(                                     \
        O, np, xp, yp, zp, uxp, uyp, uzp, gaminv, ex, ey, ez, bx, by, bz, xmin, ymin,     \
        zmin, dx, dy, dz, dtt, nx, ny, nz, nxguard, nyguard, nzguard, exg, eyg, ezg, bxg, \
        byg, bzg, q, m, lvect, l_lower_order_in_v, dt, particle_pusher, clight, stream);  \
  }
PXRB_FGP_N(1)
PXRB_FGP_N(2)
PXRB_FGP_N(3)
#undef PXRB_FGP_N

int pxrb_geteb3d_energy_conserving(
    int64_t np, const double* xp, const double* yp, const double* zp, double* ex, double* ey,
    double* ez, double* bx, double* by, double* bz, double xmin, double ymin, double zmin,
    double dx, double dy, double dz, int64_t nx, int64_t ny, int64_t nz, int64_t nxguard,
    int64_t nyguard, int64_t nzguard, int64_t nox, int64_t noy, int64_t noz,
    const double* exg, const double* eyg, const double* ezg, const double* bxg,
    const double* byg, const double* bzg, int64_t ll4symtry, int64_t l_lower_order_in_v,
    int64_t lvect, int64_t field_gathe_algo, int64_t l_nodal, void* stream) {
  (void)lvect; (void)field_gathe_algo;
  if (np < 0) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  if (nox != noy || noy != noz || nox < 1 || nox > 3 || ll4symtry) return PXRB_EUNSUPPORTED;
  const void* ptrs[] = {xp, yp, zp, ex, ey, ez, bx, by, bz, exg, eyg, ezg, bxg, byg, bzg};
  for (const void* p : ptrs) if (bad_ptr(p)) return PXRB_EINVAL;
  GEBParams p;
  p.np = np; p.xp = xp; p.yp = yp; p.zp = zp;
  p.ex = ex; p.ey = ey; p.ez = ez; p.bx = bx; p.by = by; p.bz = bz;
  p.xmin = xmin; p.ymin = ymin; p.zmin = zmin;
  p.dxi = 1.0 / dx; p.dyi = 1.0 / dy; p.dzi = 1.0 / dz;
  p.exg = exg; p.eyg = eyg; p.ezg = ezg; p.bxg = bxg; p.byg = byg; p.bzg = bzg;
  p.G = make_grid(nx, ny, nz, nxguard, nyguard, nzguard);
  p.order = (int)nox; p.lower = l_lower_order_in_v != 0;
  p.ss = l_nodal ? 0.0 : 0.5;
  k_geteb<<<nblocks(np), TPB, 0, (cudaStream_t)stream>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

static int launch_push(int kind, int64_t np, double* ux, double* uy, double* uz, double* gi,
                       const double* ex, const double* ey, const double* ez,
                       const double* bx, const double* by, const double* bz, double* x,
                       double* y, double* z, double q, double m, double dt, double clight,
                       int which, void* stream) {
  if (np < 0) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  PushParams p;
  p.np = np; p.ux = ux; p.uy = uy; p.uz = uz; p.gi = gi;
  p.ex = ex; p.ey = ey; p.ez = ez; p.bx = bx; p.by = by; p.bz = bz;
  p.x = x; p.y = y; p.z = z; p.q = q; p.m = m; p.dt = dt; p.clight = clight; p.which = which;
  cudaStream_t s = (cudaStream_t)stream;
  int nb = grid_stride_blocks(np);
  switch (kind) {
    case 0: k_boris<<<nb, TPB, 0, s>>>(p); break;
    case 1: k_vay<<<nb, TPB, 0, s>>>(p); break;
    case 2: k_set_gamma<<<nb, TPB, 0, s>>>(p); break;
    case 3: k_pushxyz<<<nb, TPB, 0, s>>>(p); break;
  }
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_boris_push_u_3d(int64_t np, double* uxp, double* uyp, double* uzp, double* gaminv,
                         const double* ex, const double* ey, const double* ez,
                         const double* bx, const double* by, const double* bz, double q,
                         double m, double dt, double clight, void* stream) {
  if (np > 0 && (!uxp || !uyp || !uzp || !gaminv || !ex || !ey || !ez || !bx || !by || !bz))
    return PXRB_EINVAL;
  return launch_push(0, np, uxp, uyp, uzp, gaminv, ex, ey, ez, bx, by, bz, nullptr, nullptr,
                     nullptr, q, m, dt, clight, 0, stream);
}

int pxrb_ebcancelpush3d(int64_t np, double* uxp, double* uyp, double* uzp, double* gi,
                        const double* ex, const double* ey, const double* ez,
                        const double* bx, const double* by, const double* bz, double q,
                        double m, double dt, int64_t which, double clight, void* stream) {
  if (which < 0 || which > 2) return PXRB_EUNSUPPORTED;
  if (np > 0 && (!uxp || !uyp || !uzp || !gi || !ex || !ey || !ez || !bx || !by || !bz))
    return PXRB_EINVAL;
  return launch_push(1, np, uxp, uyp, uzp, gi, ex, ey, ez, bx, by, bz, nullptr, nullptr,
                     nullptr, q, m, dt, clight, (int)which, stream);
}

int pxrb_set_gamma(int64_t np, const double* uxp, const double* uyp, const double* uzp,
                   double* gaminv, double clight, void* stream) {
  if (np > 0 && (!uxp || !uyp || !uzp || !gaminv)) return PXRB_EINVAL;
  return launch_push(2, np, const_cast<double*>(uxp), const_cast<double*>(uyp),
                     const_cast<double*>(uzp), gaminv, nullptr, nullptr, nullptr, nullptr,
                     nullptr, nullptr, nullptr, nullptr, nullptr, 0, 1, 0, clight, 0, stream);
}

int pxrb_pushxyz(int64_t np, double* xp, double* yp, double* zp, const double* uxp,
                 const double* uyp, const double* uzp, const double* gaminv, double dt,
                 void* stream) {
  if (np > 0 && (!xp || !yp || !zp || !uxp || !uyp || !uzp || !gaminv)) return PXRB_EINVAL;
  return launch_push(3, np, const_cast<double*>(uxp), const_cast<double*>(uyp),
                     const_cast<double*>(uzp), const_cast<double*>(gaminv), nullptr, nullptr,
                     nullptr, nullptr, nullptr, nullptr, xp, yp, zp, 0, 1, dt, 1, 0, stream);
}

int pxrb_depose_jxjyjz(double* jx, double* jy, double* jz, int64_t np, const double* xp,
                       const double* yp, const double* zp, const double* uxp,
                       const double* uyp, const double* uzp, const double* gaminv,
                       const double* w, double q, double xmin, double ymin, double zmin,
                       double dt, double dx, double dy, double dz, int64_t nx, int64_t ny,
                       int64_t nz, int64_t nxguard, int64_t nyguard, int64_t nzguard,
                       int64_t nox, int64_t noy, int64_t noz, int64_t current_depo_algo,
                       int* err_flag, void* stream) {
  if (np < 0) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  if (nox != noy || noy != noz || nox < 1 || nox > 3) return PXRB_EUNSUPPORTED;
  if (current_depo_algo != 0 && current_depo_algo != 1) return PXRB_EUNSUPPORTED;
  const void* ptrs[] = {jx, jy, jz, xp, yp, zp, uxp, uyp, uzp, gaminv, w, err_flag};
  for (const void* p : ptrs) if (bad_ptr(p)) return PXRB_EINVAL;
  DepParams p;
  p.np = np; p.xp = xp; p.yp = yp; p.zp = zp; p.uxp = uxp; p.uyp = uyp; p.uzp = uzp;
  p.gaminv = gaminv; p.w = w; p.jx = jx; p.jy = jy; p.jz = jz;
  p.G = make_grid(nx, ny, nz, nxguard, nyguard, nzguard);
  p.q = q; p.xmin = xmin; p.ymin = ymin; p.zmin = zmin;
  p.dxi = 1.0 / dx; p.dyi = 1.0 / dy; p.dzi = 1.0 / dz;
  p.dtsdx = dt * p.dxi; p.dtsdy = dt * p.dyi; p.dtsdz = dt * p.dzi;
  p.invdtdx = 1.0 / (dt * dy * dz); p.invdtdy = 1.0 / (dt * dx * dz);
  p.invdtdz = 1.0 / (dt * dx * dy);
  p.reconstruct = current_depo_algo == 1;
  p.err = err_flag;
  cudaStream_t s = (cudaStream_t)stream;
  int nb = nblocks(np);
  if (nox == 1) k_esirkepov<1><<<nb, TPB, 0, s>>>(p);
  else if (nox == 2) k_esirkepov<2><<<nb, TPB, 0, s>>>(p);
  else k_esirkepov<3><<<nb, TPB, 0, s>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_depose_rho(int64_t order, double* rho, int64_t np, const double* xp,
                    const double* yp, const double* zp, const double* w, double q,
                    double xmin, double ymin, double zmin, double dx, double dy, double dz,
                    int64_t nx, int64_t ny, int64_t nz, int64_t nxguard, int64_t nyguard,
                    int64_t nzguard, void* stream) {
  if (np < 0) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  if (order < 1 || order > 3) return PXRB_EUNSUPPORTED;
  if (!rho || !xp || !yp || !zp || !w) return PXRB_EINVAL;
  RhoParams p;
  p.np = np; p.xp = xp; p.yp = yp; p.zp = zp; p.w = w; p.rho = rho;
  p.G = make_grid(nx, ny, nz, nxguard, nyguard, nzguard);
  p.q = q; p.xmin = xmin; p.ymin = ymin; p.zmin = zmin;
  p.dxi = 1.0 / dx; p.dyi = 1.0 / dy; p.dzi = 1.0 / dz;
  p.invvol = p.dxi * p.dyi * p.dzi;
  cudaStream_t s = (cudaStream_t)stream;
  int nb = nblocks(np);
  if (order == 1) k_rho<1><<<nb, TPB, 0, s>>>(p);
  else if (order == 2) k_rho<2><<<nb, TPB, 0, s>>>(p);
  else k_rho<3><<<nb, TPB, 0, s>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

static GridG grid_lohi(const int64_t* lo, const int64_t* hi) {
  GridG g;
  // An array with Fortran bounds (lo:hi) per axis as a guarded grid: guards
  // gx = -lo, so that idx(i) = i - lo; and nx = hi + lo, so that the extent
  // nx + 1 + 2 gx equals hi - lo + 1.
  g.gx = -lo[0]; g.gy = -lo[1]; g.gz = -lo[2];
  g.nx = hi[0] + lo[0]; g.ny = hi[1] + lo[1]; g.nz = hi[2] + lo[2];
  g.sx = hi[0] - lo[0] + 1;
  g.sy = g.sx * (hi[1] - lo[1] + 1);
  return g;
}

static int yee_setup(YeeParams& p, const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                     const int64_t* yhi, const int64_t* zlo, const int64_t* zhi) {
  const int64_t* L[3] = {xlo, ylo, zlo};
  const int64_t* H[3] = {xhi, yhi, zhi};
  for (int a = 0; a < 3; ++a) { p.ulo[a] = 1 << 30; p.uhi[a] = -(1 << 30); }
  for (int c = 0; c < 3; ++c)
    for (int a = 0; a < 3; ++a) {
      p.lo[c][a] = (int)L[c][a]; p.hi[c][a] = (int)H[c][a];
      p.ulo[a] = p.lo[c][a] < p.ulo[a] ? p.lo[c][a] : p.ulo[a];
      p.uhi[a] = p.hi[c][a] > p.uhi[a] ? p.hi[c][a] : p.uhi[a];
    }
  for (int a = 0; a < 3; ++a) if (p.uhi[a] < p.ulo[a]) return 1;
  return 0;
}

int pxrb_push_em3d_evec(const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                        const int64_t* yhi, const int64_t* zlo, const int64_t* zhi,
                        double* ex, const int64_t* exlo, const int64_t* exhi, double* ey,
                        const int64_t* eylo, const int64_t* eyhi, double* ez,
                        const int64_t* ezlo, const int64_t* ezhi, const double* bx,
                        const int64_t* bxlo, const int64_t* bxhi, const double* by,
                        const int64_t* bylo, const int64_t* byhi, const double* bz,
                        const int64_t* bzlo, const int64_t* bzhi, const double* jx,
                        const int64_t* jxlo, const int64_t* jxhi, const double* jy,
                        const int64_t* jylo, const int64_t* jyhi, const double* jz,
                        const int64_t* jzlo, const int64_t* jzhi, double mudt, double dtsdx,
                        double dtsdy, double dtsdz, void* stream) {
  if (!ex || !ey || !ez || !bx || !by || !bz || !jx || !jy || !jz) return PXRB_EINVAL;
  YeeParams p;
  if (yee_setup(p, xlo, xhi, ylo, yhi, zlo, zhi)) return PXRB_OK;  // empty ranges
  p.ex = ex; p.ey = ey; p.ez = ez;
  p.bx = const_cast<double*>(bx); p.by = const_cast<double*>(by); p.bz = const_cast<double*>(bz);
  p.jx = jx; p.jy = jy; p.jz = jz;
  p.gex = grid_lohi(exlo, exhi); p.gey = grid_lohi(eylo, eyhi); p.gez = grid_lohi(ezlo, ezhi);
  p.gbx = grid_lohi(bxlo, bxhi); p.gby = grid_lohi(bylo, byhi); p.gbz = grid_lohi(bzlo, bzhi);
  p.gjx = grid_lohi(jxlo, jxhi); p.gjy = grid_lohi(jylo, jyhi); p.gjz = grid_lohi(jzlo, jzhi);
  p.mudt = mudt; p.dtsdx = dtsdx; p.dtsdy = dtsdy; p.dtsdz = dtsdz;
  dim3 blk(32, 8, 1);
  dim3 grd((p.uhi[0] - p.ulo[0] + 1 + 31) / 32, (p.uhi[1] - p.ulo[1] + 1 + 7) / 8,
           p.uhi[2] - p.ulo[2] + 1);
  k_yee_e<<<grd, blk, 0, (cudaStream_t)stream>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_push_em3d_bvec(const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                        const int64_t* yhi, const int64_t* zlo, const int64_t* zhi,
                        const double* ex, const int64_t* exlo, const int64_t* exhi,
                        const double* ey, const int64_t* eylo, const int64_t* eyhi,
                        const double* ez, const int64_t* ezlo, const int64_t* ezhi,
                        double* bx, const int64_t* bxlo, const int64_t* bxhi, double* by,
                        const int64_t* bylo, const int64_t* byhi, double* bz,
                        const int64_t* bzlo, const int64_t* bzhi, double dtsdx, double dtsdy,
                        double dtsdz, void* stream) {
  if (!ex || !ey || !ez || !bx || !by || !bz) return PXRB_EINVAL;
  YeeParams p;
  if (yee_setup(p, xlo, xhi, ylo, yhi, zlo, zhi)) return PXRB_OK;
  p.ex = const_cast<double*>(ex); p.ey = const_cast<double*>(ey); p.ez = const_cast<double*>(ez);
  p.bx = bx; p.by = by; p.bz = bz;
  p.jx = p.jy = p.jz = nullptr;
  p.gex = grid_lohi(exlo, exhi); p.gey = grid_lohi(eylo, eyhi); p.gez = grid_lohi(ezlo, ezhi);
  p.gbx = grid_lohi(bxlo, bxhi); p.gby = grid_lohi(bylo, byhi); p.gbz = grid_lohi(bzlo, bzhi);
  p.mudt = 0; p.dtsdx = dtsdx; p.dtsdy = dtsdy; p.dtsdz = dtsdz;
  dim3 blk(32, 8, 1);
  dim3 grd((p.uhi[0] - p.ulo[0] + 1 + 31) / 32, (p.uhi[1] - p.ulo[1] + 1 + 7) / 8,
           p.uhi[2] - p.ulo[2] + 1);
  k_yee_b<<<grd, blk, 0, (cudaStream_t)stream>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

static int bc_launch(double** arrs, int na, int64_t nx, int64_t ny, int64_t nz, int64_t nxg,
                     int64_t nyg, int64_t nzg, int mode, void* stream) {
  if (na < 1 || na > 3) return PXRB_EINVAL;
  for (int q = 0; q < na; ++q) if (!arrs[q]) return PXRB_EINVAL;
  // an axis of no cells and no guards (ny = 0 of PICSAR's x-z grids) is skipped
  auto bad = [](int64_t n, int64_t g) { return g < 0 || (n <= g && !(n == 0 && g == 0)); };
  if (bad(nx, nxg) || bad(ny, nyg) || bad(nz, nzg)) return PXRB_ERANGE;
  BcParams p;
  for (int q = 0; q < 3; ++q) p.a[q] = q < na ? arrs[q] : nullptr;
  p.na = na; p.G = make_grid(nx, ny, nz, nxg, nyg, nzg); p.mode = mode;
  i64 ext[3] = {nx + 1 + 2 * nxg, ny + 1 + 2 * nyg, nz + 1 + 2 * nzg};
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nn[3] = {nx, ny, nz}, gg[3] = {nxg, nyg, nzg};
  for (int ax = 0; ax < 3; ++ax) {
    if (nn[ax] == 0 && gg[ax] == 0) continue;
    p.axis = ax;
    i64 nlines = ext[(ax + 1) % 3] * ext[(ax + 2) % 3];
    k_bc_axis<<<nblocks(nlines, 128), 128, 0, s>>>(p);
  }
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_field_bc_periodic(double* f1, double* f2, double* f3, int64_t nx, int64_t ny,
                           int64_t nz, int64_t nxg, int64_t nyg, int64_t nzg, void* stream) {
  double* a[3] = {f1, f2, f3};
  int na = f3 ? 3 : (f2 ? 2 : 1);
  return bc_launch(a, na, nx, ny, nz, nxg, nyg, nzg, 0, stream);
}

int pxrb_summation_bcs_periodic(double* f1, double* f2, double* f3, int64_t nx, int64_t ny,
                                int64_t nz, int64_t nxg, int64_t nyg, int64_t nzg,
                                void* stream) {
  double* a[3] = {f1, f2, f3};
  int na = f3 ? 3 : (f2 ? 2 : 1);
  int rc = bc_launch(a, na, nx, ny, nz, nxg, nyg, nzg, 1, stream);
  if (rc) return rc;
  return bc_launch(a, na, nx, ny, nz, nxg, nyg, nzg, 0, stream);
}

int pxrb_geteb2dxz_energy_conserving(
    int64_t np, const double* xp, const double* yp, const double* zp, double* ex, double* ey,
    double* ez, double* bx, double* by, double* bz, double xmin, double ymin, double zmin,
    double dx, double dy, double dz, int64_t nx, int64_t ny, int64_t nz, int64_t nxguard,
    int64_t nyguard, int64_t nzguard, int64_t nox, int64_t noy, int64_t noz,
    const double* exg, const double* eyg, const double* ezg, const double* bxg,
    const double* byg, const double* bzg, int64_t l4symtry, int64_t l_lower_order_in_v,
    int64_t lvect, int64_t field_gathe_algo, int64_t l_nodal, void* stream) {
  (void)yp; (void)ymin; (void)dy; (void)ny; (void)nyguard; (void)noy; (void)lvect;
  (void)field_gathe_algo;
  if (np < 0) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  if (nox != noz || nox < 1 || nox > 3 || l4symtry) return PXRB_EUNSUPPORTED;
  if (!xp || !zp || !ex || !ey || !ez || !bx || !by || !bz || !exg || !eyg || !ezg || !bxg ||
      !byg || !bzg)
    return PXRB_EINVAL;
  GEB2Params p;
  p.np = np; p.xp = xp; p.zp = zp;
  p.ex = ex; p.ey = ey; p.ez = ez; p.bx = bx; p.by = by; p.bz = bz;
  p.xmin = xmin; p.zmin = zmin; p.dxi = 1.0 / dx; p.dzi = 1.0 / dz;
  p.exg = exg; p.eyg = eyg; p.ezg = ezg; p.bxg = bxg; p.byg = byg; p.bzg = bzg;
  p.G.gx = nxguard; p.G.gz = nzguard; p.G.sx = nx + 1 + 2 * nxguard;
  p.order = (int)nox; p.lower = l_lower_order_in_v ? 1 : 0;
  p.ss = l_nodal ? 0.0 : 0.5;
  k_geteb2d<<<nblocks(np), TPB, 0, (cudaStream_t)stream>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_depose_jxjyjz_2d(double* jx, double* jy, double* jz, int64_t np, const double* xp,
                          const double* yp, const double* zp, const double* uxp,
                          const double* uyp, const double* uzp, const double* gaminv,
                          const double* w, double q, double xmin, double zmin, double dt,
                          double dx, double dz, int64_t nx, int64_t nz, int64_t nxguard,
                          int64_t nzguard, int64_t nox, int64_t noz, int64_t lvect,
                          void* stream) {
  (void)yp; (void)lvect;
  if (np < 0) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  if (nox != noz || nox < 1 || nox > 3) return PXRB_EUNSUPPORTED;
  if (!jx || !jy || !jz || !xp || !zp || !uxp || !uyp || !uzp || !gaminv || !w)
    return PXRB_EINVAL;
  Dep2Params p;
  p.np = np; p.jx = jx; p.jy = jy; p.jz = jz;
  p.xp = xp; p.zp = zp; p.uxp = uxp; p.uyp = uyp; p.uzp = uzp; p.gaminv = gaminv; p.w = w;
  p.q = q; p.xmin = xmin; p.zmin = zmin; p.dt = dt; p.dx = dx; p.dz = dz;
  p.G.gx = nxguard; p.G.gz = nzguard; p.G.sx = nx + 1 + 2 * nxguard;
  cudaStream_t s = (cudaStream_t)stream;
  if (nox == 1) k_esirkepov2d<1><<<nblocks(np), TPB, 0, s>>>(p);
  else if (nox == 2) k_esirkepov2d<2><<<nblocks(np), TPB, 0, s>>>(p);
  else k_esirkepov2d<3><<<nblocks(np), TPB, 0, s>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

static int yee2d_setup(Yee2Params& p, const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                       const int64_t* yhi, const int64_t* zlo, const int64_t* zhi) {
  const int64_t* L[3] = {xlo, ylo, zlo};
  const int64_t* H[3] = {xhi, yhi, zhi};
  for (int a = 0; a < 2; ++a) { p.ulo[a] = 1 << 30; p.uhi[a] = -(1 << 30); }
  for (int c = 0; c < 3; ++c)
    for (int a = 0; a < 2; ++a) {
      p.lo[c][a] = (int)L[c][a]; p.hi[c][a] = (int)H[c][a];
      p.ulo[a] = p.lo[c][a] < p.ulo[a] ? p.lo[c][a] : p.ulo[a];
      p.uhi[a] = p.hi[c][a] > p.uhi[a] ? p.hi[c][a] : p.uhi[a];
    }
  for (int a = 0; a < 2; ++a) if (p.uhi[a] < p.ulo[a]) return 1;
  return 0;
}

int pxrb_push_em2d_evec(const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                        const int64_t* yhi, const int64_t* zlo, const int64_t* zhi,
                        double* ex, const int64_t* exlo, const int64_t* exhi, double* ey,
                        const int64_t* eylo, const int64_t* eyhi, double* ez,
                        const int64_t* ezlo, const int64_t* ezhi, const double* bx,
                        const int64_t* bxlo, const int64_t* bxhi, const double* by,
                        const int64_t* bylo, const int64_t* byhi, const double* bz,
                        const int64_t* bzlo, const int64_t* bzhi, const double* jx,
                        const int64_t* jxlo, const int64_t* jxhi, const double* jy,
                        const int64_t* jylo, const int64_t* jyhi, const double* jz,
                        const int64_t* jzlo, const int64_t* jzhi, double mudt, double dtsdx,
                        double dtsdy, double dtsdz, void* stream) {
  (void)dtsdy;
  if (!ex || !ey || !ez || !bx || !by || !bz || !jx || !jy || !jz) return PXRB_EINVAL;
  Yee2Params p;
  if (yee2d_setup(p, xlo, xhi, ylo, yhi, zlo, zhi)) return PXRB_OK;
  p.ex = ex; p.ey = ey; p.ez = ez;
  p.bx = const_cast<double*>(bx); p.by = const_cast<double*>(by); p.bz = const_cast<double*>(bz);
  p.jx = jx; p.jy = jy; p.jz = jz;
  p.gex = g2_lohi(exlo, exhi); p.gey = g2_lohi(eylo, eyhi); p.gez = g2_lohi(ezlo, ezhi);
  p.gbx = g2_lohi(bxlo, bxhi); p.gby = g2_lohi(bylo, byhi); p.gbz = g2_lohi(bzlo, bzhi);
  p.gjx = g2_lohi(jxlo, jxhi); p.gjy = g2_lohi(jylo, jyhi); p.gjz = g2_lohi(jzlo, jzhi);
  p.mudt = mudt; p.dtsdx = dtsdx; p.dtsdz = dtsdz;
  dim3 blk(32, 8, 1);
  dim3 grd((p.uhi[0] - p.ulo[0] + 1 + 31) / 32, (p.uhi[1] - p.ulo[1] + 1 + 7) / 8, 1);
  k_yee2d_e<<<grd, blk, 0, (cudaStream_t)stream>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_push_em2d_bvec(const int64_t* xlo, const int64_t* xhi, const int64_t* ylo,
                        const int64_t* yhi, const int64_t* zlo, const int64_t* zhi,
                        const double* ex, const int64_t* exlo, const int64_t* exhi,
                        const double* ey, const int64_t* eylo, const int64_t* eyhi,
                        const double* ez, const int64_t* ezlo, const int64_t* ezhi,
                        double* bx, const int64_t* bxlo, const int64_t* bxhi, double* by,
                        const int64_t* bylo, const int64_t* byhi, double* bz,
                        const int64_t* bzlo, const int64_t* bzhi, double dtsdx, double dtsdy,
                        double dtsdz, void* stream) {
  (void)dtsdy;
  if (!ex || !ey || !ez || !bx || !by || !bz) return PXRB_EINVAL;
  Yee2Params p;
  if (yee2d_setup(p, xlo, xhi, ylo, yhi, zlo, zhi)) return PXRB_OK;
  p.ex = const_cast<double*>(ex); p.ey = const_cast<double*>(ey); p.ez = const_cast<double*>(ez);
  p.bx = bx; p.by = by; p.bz = bz;
  p.jx = p.jy = p.jz = nullptr;
  p.gex = g2_lohi(exlo, exhi); p.gey = g2_lohi(eylo, eyhi); p.gez = g2_lohi(ezlo, ezhi);
  p.gbx = g2_lohi(bxlo, bxhi); p.gby = g2_lohi(bylo, byhi); p.gbz = g2_lohi(bzlo, bzhi);
  p.mudt = 0; p.dtsdx = dtsdx; p.dtsdz = dtsdz;
  dim3 blk(32, 8, 1);
  dim3 grd((p.uhi[0] - p.ulo[0] + 1 + 31) / 32, (p.uhi[1] - p.ulo[1] + 1 + 7) / 8, 1);
  k_yee2d_b<<<grd, blk, 0, (cudaStream_t)stream>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_pushxz(int64_t np, double* xp, double* zp, const double* uxp, const double* uzp,
                const double* gaminv, double dt, void* stream) {
  if (np < 0) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  if (!xp || !zp || !uxp || !uzp || !gaminv) return PXRB_EINVAL;
  k_pushxz<<<nblocks(np), TPB, 0, (cudaStream_t)stream>>>(np, xp, zp, uxp, uzp, gaminv, dt);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

int pxrb_particle_bcs_periodic(int64_t np, double* xp, double* yp, double* zp, double xmin,
                               double ymin, double zmin, double xmax, double ymax,
                               double zmax, void* stream) {
  if (np < 0) return PXRB_EINVAL;
  if (np == 0) return PXRB_OK;
  if (!xp || !yp || !zp) return PXRB_EINVAL;
  WrapParams p;
  p.np = np; p.x = xp; p.y = yp; p.z = zp;
  p.lo[0] = xmin; p.lo[1] = ymin; p.lo[2] = zmin;
  p.hi[0] = xmax; p.hi[1] = ymax; p.hi[2] = zmax;
  k_wrap<<<grid_stride_blocks(np), TPB, 0, (cudaStream_t)stream>>>(p);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

}  // extern "C"
